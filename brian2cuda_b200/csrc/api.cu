// Host runtime of libb2b: the C ABI of include/b2b.h.
//
// Plays the role of brian2cuda's generated project scaffold (templates/objects.cu array
// management, templates/network.cu step loop, templates/rand.cu buffers) for the hot path,
// but as a library: the network is described once, laid out on the GPU by b2b_finalize,
// and advanced by replaying a CUDA graph of `steps_per_graph` steps per launch with no host
// synchronisation inside a run.
#include <dlfcn.h>

#include <algorithm>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <new>
#include <numeric>

#include "b2b_build.h"
#include "b2b_internal.h"

using namespace b2b;

namespace {

b2b_status fail(b2b_net* net, b2b_status code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (net) net->err = buf;
  return code;
}

#define CU(call)                                                                          \
  do {                                                                                    \
    cudaError_t _e = (call);                                                              \
    if (_e != cudaSuccess)                                                                \
      return fail(net, B2B_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(_e));     \
  } while (0)

#define CHECK(cond, code, ...)                       \
  do {                                               \
    if (!(cond)) return fail(net, code, __VA_ARGS__); \
  } while (0)

#define GUARD_BEGIN try {
#define GUARD_END                                                     \
  }                                                                   \
  catch (const std::bad_alloc&) {                                     \
    return fail(net, B2B_ERR_OOM, "host allocation failed");          \
  }

size_t var_size(int dtype, int var) {
  if (var == B2B_VAR_NOT_REFRACTORY) return 1;
  return dtype == B2B_F32 ? 4 : 8;
}
size_t real_size(int dtype) { return dtype == B2B_F32 ? 4 : 8; }

// model_vars: state variables of a generated model (KIND_MODEL), slots 0 .. model_vars-1.
bool kind_has_var(int kind, int var, int model_vars = 0) {
  switch (kind) {
    case KIND_LIF:
      return var == B2B_VAR_V || var == B2B_VAR_GE || var == B2B_VAR_GI ||
             var == B2B_VAR_LASTSPIKE || var == B2B_VAR_NOT_REFRACTORY;
    case KIND_HH:
      return var >= 0 && var < kMaxVars;
    case KIND_MODEL:
      return (var >= 0 && var < model_vars) || var == B2B_VAR_LASTSPIKE ||
             var == B2B_VAR_NOT_REFRACTORY;
    default:
      return false;
  }
}

int64_t pad_to(int64_t n, int64_t q) { return (n + q - 1) / q * q; }

// Brian2's timestep(t, dt) on the host.
int64_t timestep_host(double t, double dt) { return (int64_t)((t + 1e-3 * dt) / dt); }

template <typename T>
cudaError_t dalloc(Pop& pop, T** p, size_t count) {
  cudaError_t e = cudaMalloc((void**)p, sizeof(T) * (count ? count : 1));
  if (e == cudaSuccess) pop.allocs.push_back(*p);
  return e;
}
template <typename T>
cudaError_t dalloc(Proj& pr, T** p, size_t count) {
  cudaError_t e = cudaMalloc((void**)p, sizeof(T) * (count ? count : 1));
  if (e == cudaSuccess) pr.allocs.push_back(*p);
  return e;
}

void put_real(std::vector<uint8_t>& buf, int dtype, int64_t i, double v) {
  if (dtype == B2B_F32) reinterpret_cast<float*>(buf.data())[i] = (float)v;
  else reinterpret_cast<double*>(buf.data())[i] = v;
}

LifDev lif_dev(const Group& g, double dt) {
  const b2b_lif_params& p = g.lif;
  LifDev d{};
  const bool leak = std::isfinite(p.taum) && p.taum > 0;
  d.A = leak ? std::exp(-dt / p.taum) : 1.0;
  d.De = p.taue > 0 ? std::exp(-dt / p.taue) : 0.0;
  d.Di = p.taui > 0 ? std::exp(-dt / p.taui) : 0.0;
  auto coupling = [&](double k, double tau, double D) {
    if (k == 0.0 || !leak) return 0.0;
    if (tau == p.taum) return k * (dt / p.taum) * d.A;
    return k * tau / (tau - p.taum) * (D - d.A);
  };
  d.Be = coupling(p.ke, p.taue, d.De);
  d.Bi = coupling(p.ki, p.taui, d.Di);
  d.El = p.El;
  d.Vt = p.Vt;
  d.Vr = p.Vr;
  d.ref_steps = p.refractory > 0 ? timestep_host(p.refractory, dt) : -1;
  d.offset = g.offset;
  d.n = g.n;
  d.has_threshold = p.has_threshold;
  d.has_reset = p.has_reset;
  d.unless_refractory = p.unless_refractory;
  return d;
}

HhDev hh_dev(const Group& g, double dt) {
  const b2b_hh_params& p = g.hh;
  HhDev d{};
  d.Cm = p.Cm; d.inv_Cm = 1.0 / p.Cm; d.gl = p.gl; d.El = p.El; d.EK = p.EK; d.ENa = p.ENa; d.gNa = p.gNa;
  d.gK = p.gK; d.VT = p.VT; d.Ee = p.Ee; d.Ei = p.Ei;
  d.De = p.taue > 0 ? std::exp(-dt / p.taue) : 0.0;
  d.Di = p.taui > 0 ? std::exp(-dt / p.taui) : 0.0;
  d.Vthr = p.Vthr;
  d.ref_steps = p.refractory > 0 ? timestep_host(p.refractory, dt) : -1;
  d.offset = g.offset;
  d.n = g.n;
  d.f = HhFloat{(float)d.Cm, (float)d.gl, (float)d.El, (float)d.EK, (float)d.ENa, (float)d.gNa,
                (float)d.gK, (float)d.VT, (float)d.Ee, (float)d.Ei, (float)d.De, (float)d.Di,
                (float)d.Vthr, (float)d.inv_Cm};
  return d;
}

bool has_refractory(const Group& g) {
  if (g.kind == KIND_LIF) return g.lif.refractory > 0;
  if (g.kind == KIND_HH) return g.hh.refractory > 0;
  if (g.kind == KIND_MODEL) return g.model_refractory > 0;
  return false;
}

b2b_status check_net(b2b_net* net) {
  if (!net) return B2B_ERR_INVALID_ARG;
  cudaError_t e = cudaSetDevice(net->cfg.device);
  if (e != cudaSuccess) return fail(net, B2B_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
  return B2B_OK;
}

b2b_status add_group(b2b_net* net, Group&& g, int32_t* gid) {
  CHECK(!net->finalized, B2B_ERR_STATE, "groups must be added before b2b_finalize");
  CHECK(gid != nullptr, B2B_ERR_INVALID_ARG, "gid is NULL");
  CHECK(g.n > 0 && g.n < ((int64_t)1 << 31) - 4096, B2B_ERR_INVALID_ARG, "bad group size %lld",
        (long long)g.n);
  CHECK(g.dtype == B2B_F32 || g.dtype == B2B_F64, B2B_ERR_INVALID_ARG, "bad dtype %d", g.dtype);
  g.staged.resize(kMaxVars);
  net->groups.push_back(std::move(g));
  *gid = (int32_t)net->groups.size() - 1;
  return B2B_OK;
}

b2b_status add_syn(b2b_net* net, Syn&& s, int32_t* sid) {
  CHECK(!net->finalized, B2B_ERR_STATE, "synapses must be added before b2b_finalize");
  CHECK(sid != nullptr, B2B_ERR_INVALID_ARG, "sid is NULL");
  CHECK(s.pre_gid >= 0 && s.pre_gid < (int)net->groups.size(), B2B_ERR_INVALID_ARG,
        "bad pre group %d", s.pre_gid);
  CHECK(s.post_gid >= 0 && s.post_gid < (int)net->groups.size(), B2B_ERR_INVALID_ARG,
        "bad post group %d", s.post_gid);
  const Group& post = net->groups[s.post_gid];
  CHECK(post.kind == KIND_LIF || post.kind == KIND_HH || post.kind == KIND_MODEL,
        B2B_ERR_INVALID_ARG, "synapse targets must be LIF, HH or generated-model groups");
  CHECK(s.target_var == B2B_VAR_V || s.target_var == B2B_VAR_GE || s.target_var == B2B_VAR_GI,
        B2B_ERR_INVALID_ARG, "target variable must be v, ge or gi (slots 0-2)");
  // a generated model's synaptic targets are its first state variables (slots 0-2)
  CHECK(post.kind != KIND_MODEL || s.target_var < post.minfo.n_vars, B2B_ERR_INVALID_ARG,
        "target slot %d is not a state variable of the generated model", s.target_var);
  CHECK(s.effect == B2B_EFFECT_ADD || s.effect == B2B_EFFECT_STDP, B2B_ERR_INVALID_ARG,
        "bad effect %d", s.effect);
  net->syns.push_back(std::move(s));
  *sid = (int32_t)net->syns.size() - 1;
  return B2B_OK;
}

// ---------------------------------------------------------------------------------------
b2b_status finalize_pops(b2b_net* net) {
  const double dt = net->cfg.dt;
  // populations: one per (kind, dtype), in order of first appearance
  for (size_t gi = 0; gi < net->groups.size(); ++gi) {
    Group& g = net->groups[gi];
    int pi = -1;
    // a generated model's group is a population of its own (its kernel is the model's)
    if (g.kind != KIND_MODEL)
      for (size_t p = 0; p < net->pops.size(); ++p)
        if (net->pops[p].kind == g.kind && net->pops[p].dtype == g.dtype) pi = (int)p;
    if (pi < 0) {
      net->pops.emplace_back();
      net->pops.back().kind = g.kind;
      net->pops.back().dtype = g.dtype;
      net->pops.back().model_launch = g.model_launch;
      net->pops.back().minfo = g.minfo;
      pi = (int)net->pops.size() - 1;
    }
    Pop& pop = net->pops[pi];
    g.pop = pi;
    g.offset = pop.n;
    pop.n = pad_to(pop.n + g.n, kPad);
    pop.groups.push_back((int)gi);
  }
  // delay range and reset placement, from the synapses
  for (const Syn& s : net->syns) {
    Pop& src = net->pops[net->groups[s.pre_gid].pop];
    src.max_delay = std::max(src.max_delay, s.dmax);
    const Group& post = net->groups[s.post_gid];
    if (post.kind == KIND_LIF && post.lif.has_reset && s.target_var == B2B_VAR_V &&
        !(net->cfg.flags & B2B_NET_RESET_BEFORE_SYNAPSES))
      net->pops[post.pop].late_reset = true;
    if (post.kind == KIND_MODEL && (post.minfo.reset_mask & (1 << s.target_var)) &&
        !(net->cfg.flags & B2B_NET_RESET_BEFORE_SYNAPSES))
      net->pops[post.pop].late_reset = true;
  }
  for (size_t pi = 0; pi < net->pops.size(); ++pi) {
    Pop& pop = net->pops[pi];
    PopDev& D = pop.dev;
    D.n = pop.n;
    D.n_groups = (int32_t)pop.groups.size();
    D.ring_len = pop.max_delay + 2;
    D.late_reset = pop.late_reset ? 1 : 0;
    const size_t rs = real_size(pop.dtype);
    // state
    if (pop.kind == KIND_LIF || pop.kind == KIND_HH || pop.kind == KIND_MODEL) {
      for (int v = 0; v < kMaxVars; ++v) {
        if (!kind_has_var(pop.kind, v, pop.minfo.n_vars)) continue;
        const size_t es = var_size(pop.dtype, v);
        std::vector<uint8_t> host(es * pop.n, 0);
        for (int gi : pop.groups) {
          const Group& g = net->groups[gi];
          if (v == B2B_VAR_LASTSPIKE && has_refractory(g))
            for (int64_t i = 0; i < g.n; ++i) put_real(host, pop.dtype, g.offset + i, -1e4);
          if (v == B2B_VAR_NOT_REFRACTORY)
            std::memset(host.data() + g.offset, 1, g.n);
          if (!g.staged[v].empty())
            std::memcpy(host.data() + es * g.offset, g.staged[v].data(), g.staged[v].size());
        }
        void* d = nullptr;
        CU(dalloc(pop, (uint8_t**)&d, es * pop.n));
        CU(cudaMemcpyAsync(d, host.data(), es * pop.n, cudaMemcpyHostToDevice, net->stream));
        CU(cudaStreamSynchronize(net->stream));
        D.var[v] = d;
      }
    }
    // parameters, and the groups' inputs (TimedArray tables in the population's dtype,
    // PoissonInputs) in an array of their own
    std::vector<uint8_t> prm;
    std::vector<GroupInputs> gins;
    for (int gi : pop.groups) {
      const Group& g = net->groups[gi];
      TimedInput ta{};
      if (!g.ta.empty()) {
        std::vector<uint8_t> host(rs * g.ta.size());
        for (size_t k = 0; k < g.ta.size(); ++k) put_real(host, pop.dtype, (int64_t)k, g.ta[k]);
        uint8_t* d = nullptr;
        CU(dalloc(pop, &d, host.size()));
        CU(cudaMemcpy(d, host.data(), host.size(), cudaMemcpyHostToDevice));
        ta = TimedInput{d, g.ta_rows, g.ta_cols, g.ta_mul, g.ta_div};
      }
      pop.inputs = pop.inputs || !g.ta.empty() || !g.pins.empty();
      PoissonInputs pin{};
      pin.count = (int32_t)g.pins.size();
      pin.after_reset = (net->cfg.flags & B2B_NET_RESET_BEFORE_SYNAPSES) ? 1 : 0;
      for (size_t k = 0; k < g.pins.size(); ++k) pin.in[k] = g.pins[k];
      gins.push_back(GroupInputs{ta, pin});
      if (pop.kind == KIND_LIF) {
        LifDev d = lif_dev(g, dt);
        prm.insert(prm.end(), (uint8_t*)&d, (uint8_t*)&d + sizeof(d));
      } else if (pop.kind == KIND_HH) {
        HhDev d = hh_dev(g, dt);
        prm.insert(prm.end(), (uint8_t*)&d, (uint8_t*)&d + sizeof(d));
      } else if (pop.kind == KIND_POISSON) {
        PoissonDev d{g.rate * dt, g.offset, g.n};
        prm.insert(prm.end(), (uint8_t*)&d, (uint8_t*)&d + sizeof(d));
      } else if (pop.kind == KIND_MODEL) {
        ModelGroupDev d{g.offset, g.n,
                        has_refractory(g) ? timestep_host(g.model_refractory, dt) : -1};
        prm.insert(prm.end(), (uint8_t*)&d, (uint8_t*)&d + sizeof(d));
      }
    }
    if (!prm.empty()) {
      CU(dalloc(pop, (uint8_t**)&pop.params_dev, prm.size()));
      CU(cudaMemcpy(pop.params_dev, prm.data(), prm.size(), cudaMemcpyHostToDevice));
      D.params = pop.params_dev;
    }
    if (pop.inputs) {
      GroupInputs* d = nullptr;
      CU(dalloc(pop, &d, gins.size()));
      CU(cudaMemcpy(d, gins.data(), sizeof(GroupInputs) * gins.size(), cudaMemcpyHostToDevice));
      D.inputs = d;
    }
    // gating surrogate: every HH group of a float32 population shares one network
    if (pop.kind == KIND_HH) {
      const Group& g0 = net->groups[pop.groups[0]];
      bool any = false;
      for (int gi : pop.groups) {
        const Group& g = net->groups[gi];
        any = any || g.surr;
        CHECK(g.surr == g0.surr && g.surr_tol == g0.surr_tol && g.surr_judge == g0.surr_judge,
              B2B_ERR_UNSUPPORTED, "HH groups of one population must share one surrogate");
      }
      for (int gi : pop.groups)
        CHECK(!any || (net->groups[gi].ta.empty() && net->groups[gi].pins.empty()),
              B2B_ERR_UNSUPPORTED,
              "TimedArray and PoissonInput inputs cannot drive a population with the gating "
              "surrogate");
      if (any) {
        CHECK(pop.dtype == B2B_F32, B2B_ERR_UNSUPPORTED, "the gating surrogate is float32 only");
        CHECK(mlp_device(g0.surr) == net->cfg.device, B2B_ERR_INVALID_ARG,
              "surrogate and net are on different devices");
        pop.surr_img = mlp_image(g0.surr);
        pop.surr_tol = (float)g0.surr_tol;
        pop.surr_judge = g0.surr_judge;
        CU(dalloc(pop, &pop.surr_cnt, 2));
        CU(cudaMemset(pop.surr_cnt, 0, 2 * sizeof(unsigned long long)));
      }
    }
    if (pop.groups.size() > 1) {
      std::vector<int32_t> vg(pop.n / 4, (int32_t)pop.groups.size() - 1);
      for (size_t k = 0; k < pop.groups.size(); ++k) {
        const Group& g = net->groups[pop.groups[k]];
        const int64_t end = k + 1 < pop.groups.size()
                                ? net->groups[pop.groups[k + 1]].offset
                                : pop.n;
        for (int64_t q = g.offset / 4; q < end / 4; ++q) vg[q] = (int32_t)k;
      }
      CU(dalloc(pop, &pop.vec_group_dev, vg.size()));
      CU(cudaMemcpy(pop.vec_group_dev, vg.data(), vg.size() * 4, cudaMemcpyHostToDevice));
      D.vec_group = pop.vec_group_dev;
    }
    // spike-history ring
    CU(dalloc(pop, &D.ring_idx, (size_t)D.ring_len * pop.n));
    CU(dalloc(pop, &D.ring_cnt, (size_t)D.ring_len));
    CU(cudaMemset(D.ring_cnt, 0, sizeof(int32_t) * D.ring_len));
    // spike monitor
    int64_t cap = 0;
    for (int gi : pop.groups) cap += net->groups[gi].mon_cap;
    if (cap > 0) {
      CU(dalloc(pop, &D.mon_idx, (size_t)cap));
      CU(dalloc(pop, &D.mon_step, (size_t)cap));
      CU(dalloc(pop, &D.mon_cnt, 1));
      CU(cudaMemset(D.mon_cnt, 0, sizeof(unsigned long long)));
      D.mon_cap = cap;
    }
    // Poisson uniform buffer; a generated model's uniform and normal buffers
    const int64_t n_uni = pop.kind == KIND_POISSON ? 1
                          : (pop.kind == KIND_MODEL ? pop.minfo.n_uniform : 0);
    const int64_t n_nrm = pop.kind == KIND_MODEL ? pop.minfo.n_normal : 0;
    if (n_uni > 0 || n_nrm > 0) {
      pop.rng_steps = net->cfg.steps_per_graph;
      if (n_uni > 0) {
        CU(dalloc(pop, (uint8_t**)&pop.rng_buf, rs * pop.rng_steps * n_uni * pop.n));
        D.rng = pop.rng_buf;
      }
      if (n_nrm > 0) {
        CU(dalloc(pop, (uint8_t**)&pop.rng_normal_buf, rs * pop.rng_steps * n_nrm * pop.n));
        D.rng_normal = pop.rng_normal_buf;
      }
      if (!net->gen) {
        if (curandCreateGenerator(&net->gen, CURAND_RNG_PSEUDO_PHILOX4_32_10) !=
                CURAND_STATUS_SUCCESS ||
            curandSetPseudoRandomGeneratorSeed(net->gen, net->cfg.seed) !=
                CURAND_STATUS_SUCCESS ||
            curandSetStream(net->gen, net->stream) != CURAND_STATUS_SUCCESS)
          return fail(net, B2B_ERR_CUDA, "cuRAND generator setup failed");
      }
    }
    // spike generator entries
    if (pop.kind == KIND_SPIKEGEN) {
      std::vector<std::pair<int64_t, int32_t>> ent;
      D.sg_period = net->groups[pop.groups[0]].sg_period;
      for (int gi : pop.groups) {
        const Group& g = net->groups[gi];
        CHECK(g.sg_period == D.sg_period, B2B_ERR_UNSUPPORTED,
              "SpikeGeneratorGroups of one net must share one period");
        for (size_t k = 0; k < g.sg_idx.size(); ++k)
          ent.emplace_back(g.sg_step[k], (int32_t)(g.sg_idx[k] + g.offset));
      }
      std::stable_sort(ent.begin(), ent.end(),
                       [](const auto& a, const auto& b) { return a.first < b.first; });
      std::vector<int64_t> st(ent.size());
      std::vector<int32_t> ix(ent.size());
      for (size_t k = 0; k < ent.size(); ++k) { st[k] = ent[k].first; ix[k] = ent[k].second; }
      int64_t* dst = nullptr;
      int32_t* dix = nullptr;
      CU(dalloc(pop, &dst, st.size()));
      CU(dalloc(pop, &dix, ix.size()));
      if (!st.empty()) {
        CU(cudaMemcpy(dst, st.data(), st.size() * 8, cudaMemcpyHostToDevice));
        CU(cudaMemcpy(dix, ix.data(), ix.size() * 4, cudaMemcpyHostToDevice));
      }
      D.sg_step = dst;
      D.sg_idx = dix;
      D.sg_n = (int64_t)st.size();
    }
  }
  return B2B_OK;
}

bool same_stdp(const b2b_stdp_params& a, const b2b_stdp_params& b) {
  return a.taupre == b.taupre && a.taupost == b.taupost && a.dApre == b.dApre &&
         a.dApost == b.dApost && a.wmin == b.wmin && a.wmax == b.wmax &&
         a.pre_adds_weight == b.pre_adds_weight;
}

struct MemberTmp {
  int32_t *i = nullptr, *j = nullptr, *d = nullptr;
  void* w = nullptr;
  uint32_t *keys = nullptr, *vals = nullptr;
  int64_t* inv = nullptr;
  void release() {
    cudaFree(i); cudaFree(j); cudaFree(d); cudaFree(w); cudaFree(keys); cudaFree(vals);
    i = j = d = nullptr; w = nullptr; keys = vals = nullptr;
  }
};

b2b_status build_proj(b2b_net* net, int pj) {
  Proj& pr = net->projs[pj];
  const Pop& src = net->pops[pr.src_pop];
  const Pop& dst = net->pops[pr.dst_pop];
  const int32_t nd = pr.dmax - pr.dmin + 1;
  const int64_t nkeys = src.n * (int64_t)nd;
  cudaStream_t s = net->stream;
  CU(dalloc(pr, &pr.off, (size_t)nkeys + 1));
  CU(cudaMemsetAsync(pr.off, 0, sizeof(int64_t) * (nkeys + 1), s));
  std::vector<MemberTmp> tmp(pr.members.size());
  struct Cleanup {
    std::vector<MemberTmp>* t;
    ~Cleanup() { for (auto& m : *t) m.release(); }
  } cleanup{&tmp};
  const size_t rs = real_size(pr.dtype);
  // per-synapse weights only for STDP and host-given weights; members with different scalar
  // weights keep one weight per member
  bool need_w = pr.effect == B2B_EFFECT_STDP;
  bool member_w = false;
  for (int sid : pr.members) {
    const Syn& sy = net->syns[sid];
    if (!sy.w.empty()) need_w = true;
    if (net->syns[pr.members[0]].w_scalar != sy.w_scalar) member_w = true;
  }
  member_w = member_w && !need_w;
  // 1) upload or generate, keys, histogram
  for (size_t m = 0; m < pr.members.size(); ++m) {
    Syn& sy = net->syns[pr.members[m]];
    const Group& gpre = net->groups[sy.pre_gid];
    const Group& gpost = net->groups[sy.post_gid];
    MemberTmp& t = tmp[m];
    if (sy.generated) {
      int64_t n = 0;
      CU(generate_random_ijd(sy.pre_lo, sy.pre_hi, gpost.n, sy.p, sy.gdmin, sy.gdmax, sy.gseed,
                             &t.i, &t.j, &t.d, &n, s));
      sy.n = n;
    } else {
      CU(cudaMalloc(&t.i, 4 * std::max<int64_t>(sy.n, 1)));
      CU(cudaMalloc(&t.j, 4 * std::max<int64_t>(sy.n, 1)));
      CU(cudaMalloc(&t.d, 4 * std::max<int64_t>(sy.n, 1)));
      if (sy.n) {
        CU(cudaMemcpyAsync(t.i, sy.i.data(), 4 * sy.n, cudaMemcpyHostToDevice, s));
        CU(cudaMemcpyAsync(t.j, sy.j.data(), 4 * sy.n, cudaMemcpyHostToDevice, s));
        if (!sy.delay.empty()) {
          CU(cudaMemcpyAsync(t.d, sy.delay.data(), 4 * sy.n, cudaMemcpyHostToDevice, s));
        } else {
          std::vector<int32_t> dd(sy.n, sy.delay_scalar);
          CU(cudaMemcpyAsync(t.d, dd.data(), 4 * sy.n, cudaMemcpyHostToDevice, s));
          CU(cudaStreamSynchronize(s));
        }
      }
      if (!sy.w.empty()) {
        CU(cudaMalloc(&t.w, sy.w.size()));
        CU(cudaMemcpyAsync(t.w, sy.w.data(), sy.w.size(), cudaMemcpyHostToDevice, s));
      }
      CU(cudaMalloc(&t.inv, 8 * std::max<int64_t>(sy.n, 1)));
      pr.allocs.push_back(t.inv);
      sy.inv = t.inv;
    }
    CHECK((uint64_t)(sy.pre_hi - sy.pre_lo) * (uint64_t)nd < (1ull << 32), B2B_ERR_UNSUPPORTED,
          "pre group size x delay range exceeds 2^32");
    CHECK(sy.n < (1ll << 31), B2B_ERR_UNSUPPORTED, "more than 2^31 synapses in one Synapses");
    CU(cudaMalloc(&t.keys, 4 * std::max<int64_t>(sy.n, 1)));
    CU(cudaMalloc(&t.vals, 4 * std::max<int64_t>(sy.n, 1)));
    CU(member_keys(t.i, t.d, sy.n, sy.pre_lo, nd, pr.dmin, (gpre.offset + sy.pre_lo) * (int64_t)nd,
                   t.keys, t.vals, pr.off, s));
    pr.n_syn += sy.n;
  }
  CU(cudaStreamSynchronize(s));
  // 2) offsets
  int64_t maxb = 0;
  CU(counts_to_offsets(pr.off, nkeys, &maxb, s));
  pr.max_bundle = maxb;
  CU(dalloc(pr, &pr.post, (size_t)pr.n_syn));
  if (need_w) CU(dalloc(pr, (uint8_t**)&pr.w, rs * (size_t)pr.n_syn));
  // 3) sort + scatter
  for (size_t m = 0; m < pr.members.size(); ++m) {
    Syn& sy = net->syns[pr.members[m]];
    const Group& gpre = net->groups[sy.pre_gid];
    const Group& gpost = net->groups[sy.post_gid];
    MemberTmp& t = tmp[m];
    const int64_t key_base = (gpre.offset + sy.pre_lo) * (int64_t)nd;
    CU(cudaMemcpy(&sy.base, pr.off + key_base, 8, cudaMemcpyDeviceToHost));
    CU(member_sort_scatter(t.keys, t.vals, sy.n, (uint64_t)(sy.pre_hi - sy.pre_lo) * nd, pr.off,
                           key_base, t.j,
                           gpost.offset, t.w, pr.dtype, pr.post, need_w ? pr.w : nullptr,
                           t.inv, s));
    if (need_w && !t.w) CU(fill_value((uint8_t*)pr.w + rs * sy.base, pr.dtype, sy.n, sy.w_scalar, s));
    t.release();
  }
  CU(cudaStreamSynchronize(s));
  // device view
  ProjDev& D = pr.dev;
  D.src_ring_idx = src.dev.ring_idx;
  D.src_ring_cnt = src.dev.ring_cnt;
  D.src_n = src.n;
  D.src_ring_len = src.dev.ring_len;
  D.dmin = pr.dmin;
  D.nd = nd;
  D.chunks = (int32_t)std::max<int64_t>(1, (pr.max_bundle + kChunk - 1) / kChunk);
  D.off = pr.off;
  D.post = pr.post;
  D.w = pr.w;
  D.w_scalar = net->syns[pr.members[0]].w_scalar;
  D.target = dst.dev.var[pr.target_var];
  for (int v = 0; v < 3; ++v) D.targets[v] = dst.dev.var[v];
  D.n_mem = 1;
  if (pr.multi_target || member_w) {
    std::vector<int64_t> hi;
    std::vector<int8_t> var;
    std::vector<double> mw;
    for (int m : pr.members) {
      const Syn& sy = net->syns[m];
      hi.push_back(net->groups[sy.pre_gid].offset + sy.pre_hi);
      var.push_back((int8_t)sy.target_var);
      mw.push_back(sy.w_scalar);
    }
    int64_t* dhi = nullptr;
    int8_t* dvar = nullptr;
    CU(dalloc(pr, &dhi, hi.size()));
    CU(dalloc(pr, &dvar, var.size()));
    CU(cudaMemcpy(dhi, hi.data(), 8 * hi.size(), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(dvar, var.data(), var.size(), cudaMemcpyHostToDevice));
    D.n_mem = (int32_t)hi.size();
    D.mem_hi = dhi;
    D.mem_var = dvar;
    if (member_w) {
      double* dw = nullptr;
      CU(dalloc(pr, &dw, mw.size()));
      CU(cudaMemcpy(dw, mw.data(), 8 * mw.size(), cudaMemcpyHostToDevice));
      D.mem_w = dw;
    }
  }
  int64_t n_dst_valid = 0;
  for (int gi : dst.groups) n_dst_valid += net->groups[gi].n;
  D.aggregate = n_dst_valid < 64 ? 1 : 0;
  pr.var_mask = 0;
  for (int m : pr.members) pr.var_mask |= (uint8_t)(1u << net->syns[m].target_var);
  pr.dst_n = dst.n;
  if (pr.effect == B2B_EFFECT_STDP) {
    const b2b_stdp_params& sp = net->syns[pr.members[0]].stdp;
    CHECK(pr.n_syn < (1ll << 31), B2B_ERR_UNSUPPORTED, "STDP projection above 2^31 synapses");
    // one interleaved record per synapse; the scattered initial weights move into it
    CU(dalloc(pr, (uint8_t**)&D.syn4, 4 * rs * (size_t)pr.n_syn));
    CU(pack_stdp(pr.w, D.syn4, pr.dtype, pr.n_syn, s));
    CU(cudaStreamSynchronize(s));
    pr.allocs.erase(std::remove(pr.allocs.begin(), pr.allocs.end(), pr.w), pr.allocs.end());
    cudaFree(pr.w);
    pr.w = nullptr;
    D.w = nullptr;
    D.taupre = sp.taupre; D.taupost = sp.taupost; D.dApre = sp.dApre; D.dApost = sp.dApost;
    D.wmin = sp.wmin; D.wmax = sp.wmax; D.pre_adds_weight = sp.pre_adds_weight;
    int64_t* poff = nullptr;
    int32_t* psyn = nullptr;
    CU(dalloc(pr, &poff, (size_t)dst.n + 1));
    CU(dalloc(pr, &psyn, (size_t)pr.n_syn));
    int64_t maxp = 0;
    CU(build_post_index(pr.post, pr.n_syn, 0, dst.n, poff, psyn, &maxp, s));
    pr.max_post_bundle = maxp;
    D.post_ring_idx = dst.dev.ring_idx;
    D.post_ring_cnt = dst.dev.ring_cnt;
    D.post_src_n = dst.n;
    D.post_ring_len = dst.dev.ring_len;
    D.post_chunks = (int32_t)std::max<int64_t>(1, (maxp + kChunk - 1) / kChunk);
    D.post_off = poff;
    D.post_syn = psyn;
  }
  return B2B_OK;
}

// Additive projections with the same kernel variant share one delivery launch (retired
// projections of a delay change included); the launch shapes go back to the built-in rule.
void build_add_batches(b2b_net* net) {
  net->add_batches.clear();
  for (const Proj& pr : net->projs) {
    if (pr.effect != B2B_EFFECT_ADD) continue;
    bool placed = false;
    for (auto& b : net->add_batches) {
      const Proj& q = *b[0];
      if ((int)b.size() < kMaxProjBatch && q.dtype == pr.dtype &&
          (q.dev.w != nullptr) == (pr.dev.w != nullptr) && q.dev.aggregate == pr.dev.aggregate) {
        b.push_back(&pr);
        placed = true;
        break;
      }
    }
    if (!placed) net->add_batches.push_back({&pr});
  }
  net->add_tune.assign(net->add_batches.size(), AddTune{});  // built-in shapes until tuned
}

b2b_status finalize_projs(b2b_net* net) {
  // merge Synapses objects into projections
  for (size_t si = 0; si < net->syns.size(); ++si) {
    Syn& sy = net->syns[si];
    const Group& gpre = net->groups[sy.pre_gid];
    const Group& gpost = net->groups[sy.post_gid];
    int pj = -1;
    for (size_t p = 0; p < net->projs.size() && pj < 0; ++p) {
      Proj& pr = net->projs[p];
      // additive Synapses objects of one source population share a projection whatever
      // their target variable (one spike ring walk); STDP ones need the same target
      if (pr.src_pop != gpre.pop || pr.dst_pop != gpost.pop || pr.effect != sy.effect)
        continue;
      if (sy.effect != B2B_EFFECT_ADD && pr.target_var != sy.target_var) continue;
      if (sy.effect == B2B_EFFECT_STDP && !same_stdp(net->syns[pr.members[0]].stdp, sy.stdp))
        continue;
      bool clash = false;
      for (int m : pr.members) {
        const Syn& o = net->syns[m];
        clash |= o.pre_gid == sy.pre_gid && o.pre_lo < sy.pre_hi && sy.pre_lo < o.pre_hi;
      }
      if (!clash) pj = (int)p;
    }
    if (pj < 0) {
      net->projs.emplace_back();
      Proj& pr = net->projs.back();
      pr.src_pop = gpre.pop;
      pr.dst_pop = gpost.pop;
      pr.target_var = sy.target_var;
      pr.effect = sy.effect;
      pr.dtype = gpost.dtype;
      pr.dmin = sy.dmin;
      pr.dmax = sy.dmax;
      pj = (int)net->projs.size() - 1;
    }
    Proj& pr = net->projs[pj];
    if (pr.target_var != sy.target_var) pr.multi_target = true;
    pr.members.push_back((int)si);
    pr.dmin = std::min(pr.dmin, sy.dmin);
    pr.dmax = std::max(pr.dmax, sy.dmax);
    sy.proj = pj;
  }
  for (Proj& pr : net->projs)
    std::sort(pr.members.begin(), pr.members.end(), [&](int a, int b) {
      return net->groups[net->syns[a].pre_gid].offset + net->syns[a].pre_lo <
             net->groups[net->syns[b].pre_gid].offset + net->syns[b].pre_lo;
    });
  for (size_t p = 0; p < net->projs.size(); ++p) {
    b2b_status st = build_proj(net, (int)p);
    if (st != B2B_OK) return st;
  }
  build_add_batches(net);
  return B2B_OK;
}

// Buffers and device views of the state and rate monitors (after the populations exist).
b2b_status setup_monitors(b2b_net* net) {
  auto mal = [&](void** p, size_t bytes) -> cudaError_t {
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 1);
    if (e == cudaSuccess) net->mon_allocs.push_back(*p);
    return e;
  };
  std::vector<StateMonDev> sd;
  for (StateMon& m : net->smons) {
    const Group& g = net->groups[m.gid];
    const Pop& pop = net->pops[g.pop];
    StateMonDev& D = m.dev;
    D.es = (int32_t)var_size(pop.dtype, m.var);
    D.src = static_cast<const uint8_t*>(pop.dev.var[m.var]);
    D.n_idx = (int64_t)m.idx.size();
    D.cap = m.cap;
    D.every = m.every;
    std::vector<int64_t> rows(m.idx);
    for (int64_t& r : rows) r += g.offset;
    void *idx = nullptr, *buf = nullptr, *steps = nullptr, *cnt = nullptr, *tk = nullptr;
    CU(mal(&idx, sizeof(int64_t) * rows.size()));
    CU(mal(&buf, (size_t)D.es * (size_t)D.n_idx * (size_t)m.cap));
    CU(mal(&steps, sizeof(int64_t) * (size_t)m.cap));
    CU(mal(&cnt, sizeof(unsigned long long)));
    CU(mal(&tk, sizeof(unsigned int)));
    CU(cudaMemcpy(idx, rows.data(), sizeof(int64_t) * rows.size(), cudaMemcpyHostToDevice));
    CU(cudaMemset(cnt, 0, sizeof(unsigned long long)));
    CU(cudaMemset(tk, 0, sizeof(unsigned int)));
    D.idx = static_cast<const int64_t*>(idx);
    D.buf = static_cast<uint8_t*>(buf);
    D.steps = static_cast<int64_t*>(steps);
    D.cnt = static_cast<unsigned long long*>(cnt);
    D.ticket = static_cast<unsigned int*>(tk);
    net->smon_max_idx = std::max(net->smon_max_idx, D.n_idx);
    sd.push_back(D);
  }
  std::vector<RateMonDev> rd;
  for (RateMon& m : net->rmons) {
    const Group& g = net->groups[m.gid];
    const Pop& pop = net->pops[g.pop];
    RateMonDev& D = m.dev;
    D.ring_idx = pop.dev.ring_idx;
    D.ring_cnt = pop.dev.ring_cnt;
    D.ring_n = pop.n;
    D.ring_len = pop.dev.ring_len;
    D.lo = g.offset;
    D.hi = g.offset + g.n;
    D.whole = pop.groups.size() == 1 ? 1 : 0;
    D.cap = m.cap;
    void *buf = nullptr, *steps = nullptr, *cnt = nullptr;
    CU(mal(&buf, sizeof(int32_t) * (size_t)m.cap));
    CU(mal(&steps, sizeof(int64_t) * (size_t)m.cap));
    CU(mal(&cnt, sizeof(unsigned long long)));
    CU(cudaMemset(cnt, 0, sizeof(unsigned long long)));
    D.buf = static_cast<int32_t*>(buf);
    D.steps = static_cast<int64_t*>(steps);
    D.cnt = static_cast<unsigned long long*>(cnt);
    rd.push_back(D);
  }
  if (!sd.empty()) {
    CU(mal((void**)&net->d_smons, sizeof(StateMonDev) * sd.size()));
    CU(cudaMemcpy(net->d_smons, sd.data(), sizeof(StateMonDev) * sd.size(),
                  cudaMemcpyHostToDevice));
  }
  if (!rd.empty()) {
    CU(mal((void**)&net->d_rmons, sizeof(RateMonDev) * rd.size()));
    CU(cudaMemcpy(net->d_rmons, rd.data(), sizeof(RateMonDev) * rd.size(),
                  cudaMemcpyHostToDevice));
  }
  return B2B_OK;
}

// A small network (small.cu) runs every step of a chunk in one CTA or one thread-block
// cluster: one LIF/HH population of at most 4096 neurons (no gating surrogate) whose
// Synapses objects are all additive and target it, with the state fitting the CTA's shared
// memory.  B2B_NET_SMALL selects the path; otherwise b2b_autotune may (site kind 14).
b2b_status setup_small(b2b_net* net) {
  const int32_t flags = net->cfg.flags;
  if (flags & (B2B_NET_CHECKED | B2B_NET_TWO_LAUNCH | B2B_NET_ONE_LAUNCH)) return B2B_OK;
  if ((flags & B2B_NET_PER_STEP) && !(flags & B2B_NET_SMALL)) return B2B_OK;
  if (!net->smons.empty() || !net->rmons.empty()) return B2B_OK;  // per-step path records
  if (net->pops.size() != 1 || net->projs.size() > kMaxProjBatch) return B2B_OK;
  const Pop& pop = net->pops[0];
  if ((pop.kind != KIND_LIF && pop.kind != KIND_HH) || pop.surr_img || pop.n > 4096)
    return B2B_OK;
  for (int gi : pop.groups)
    if (!net->groups[gi].pins.empty()) return B2B_OK;   // the one-CTA kernel draws none
  SmallDev& D = net->sdev;
  D = SmallDev{};
  D.pop = pop.dev;
  D.n_proj = (int32_t)net->projs.size();
  D.nd_max = 1;
  D.warp_prefix = 1;
  for (size_t p = 0; p < net->projs.size(); ++p) {
    const Proj& pr = net->projs[p];
    if (pr.effect != B2B_EFFECT_ADD || pr.src_pop != 0 || pr.dst_pop != 0) return B2B_OK;
    for (int m : pr.members) {
      const int v = net->syns[m].target_var;
      if (v != B2B_VAR_V && v != B2B_VAR_GE && v != B2B_VAR_GI) return B2B_OK;
    }
    D.proj[p] = pr.dev;
    D.proj_target[p] = pr.target_var;
    D.nd_max = std::max<int32_t>(D.nd_max, pr.dev.nd);
    if (pr.dev.nd > 64) D.warp_prefix = 0;
  }
  if (small_smem(D, pop.kind, pop.dtype) > 200 * 1024) return B2B_OK;
  D.ring_in_smem = 1;
  if (small_smem(D, pop.kind, pop.dtype) > 200 * 1024) D.ring_in_smem = 0;
  D.cluster = 1;                 // one CTA until tuned (b2b_autotune, site kind 14)
  D.slice = pop.n;
  // the pull form: projections whose synapses have no delay (0 steps) and no weight of
  // their own; their connectivity is kept on the host to be split by slice for a cluster size
  bool pull = pop.n <= 8192;
  for (const Proj& pr : net->projs)
    pull = pull && pr.dmin == 0 && pr.dmax == 0 && pr.dev.w == nullptr && pr.n_syn < (1ll << 26);
  if (pull) {
    net->pull_host_off.assign(net->projs.size(), {});
    net->pull_host_post.assign(net->projs.size(), {});
    for (size_t p = 0; p < net->projs.size(); ++p) {
      const Proj& pr = net->projs[p];
      net->pull_host_off[p].assign(pop.n + 1, 0);
      net->pull_host_post[p].assign(std::max<int64_t>(pr.n_syn, 1), 0);
      CU(cudaMemcpy(net->pull_host_off[p].data(), pr.off, sizeof(int64_t) * (pop.n + 1),
                    cudaMemcpyDeviceToHost));
      if (pr.n_syn)
        CU(cudaMemcpy(net->pull_host_post[p].data(), pr.post, sizeof(int32_t) * pr.n_syn,
                      cudaMemcpyDeviceToHost));
    }
    net->pull_ok = true;
  }
  net->small_ok = true;
  net->small = (flags & B2B_NET_SMALL) != 0;
  return B2B_OK;
}

// Populations up to this size run the two concurrent launches unless tuned otherwise
// (measured: 1e5 HH neurons 38.6 vs 50.9 ms per simulated second).  Above it the pending
// input's read and clear (16 B per neuron and step for ge and gi in float32) costs more HBM
// time than the overlap saves: 3.9e6 HH neurons 70.1 vs 62.2 us per step.
constexpr int64_t kAutoTwoLaunchMaxNeurons = 1 << 18;

// The step as two concurrent launches (pending.cu) applies when the net is one LIF/HH
// population (no gating surrogate, no state or rate monitor) whose synapses are all additive
// onto its ge/gi with delays of at least one step.
b2b_status setup_two_launch(b2b_net* net) {
  const int32_t flags = net->cfg.flags;
  if (flags & (B2B_NET_PER_STEP | B2B_NET_SMALL)) return B2B_OK;
  if ((flags & B2B_NET_CHECKED) && !(flags & (B2B_NET_TWO_LAUNCH | B2B_NET_ONE_LAUNCH)))
    return B2B_OK;
  if (!net->smons.empty() || !net->rmons.empty()) return B2B_OK;  // per-step path records
  if (net->pops.size() != 1 || net->projs.empty() || net->projs.size() > kMaxProjBatch)
    return B2B_OK;
  const Pop& pop = net->pops[0];
  if (pop.kind != KIND_LIF && pop.kind != KIND_HH) return B2B_OK;
  if (pop.surr_img) return B2B_OK;
  int32_t nd_max = 1;
  for (const Proj& pr : net->projs) {
    if (pr.effect != B2B_EFFECT_ADD || pr.dmin < 1) return B2B_OK;
    for (int m : pr.members) {
      const int v = net->syns[m].target_var;
      if (v != B2B_VAR_GE && v != B2B_VAR_GI) return B2B_OK;
    }
    nd_max = std::max(nd_max, pr.dev.nd);
  }
  PendingDev& F = net->pdev;
  F = PendingDev{};
  F.pop = pop.dev;
  F.n_proj = (int32_t)net->projs.size();
  F.nd_max = nd_max;
  const size_t rs = real_size(pop.dtype);
  for (size_t p = 0; p < net->projs.size(); ++p) {
    const Proj& pr = net->projs[p];
    F.proj[p] = pr.dev;
    for (int m : pr.members) {
      const int v = net->syns[m].target_var;
      if (!F.acc[v]) {
        CU(cudaMalloc(&F.acc[v], 2 * rs * pop.n));
        net->pending_allocs.push_back(F.acc[v]);
        CU(cudaMemset(F.acc[v], 0, 2 * rs * pop.n));
      }
      F.proj[p].targets[v] = F.acc[v];
    }
    F.proj[p].target = F.acc[pr.target_var];
  }
  int sms = kNumSMs;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, net->cfg.device);
  F.group = 8;
  net->pending_grid = 2 * sms;
  // the update launch is the per-step neuron kernel, adding in the input that the previous
  // step's delivery left in acc
  net->fold_dev = pop.dev;
  for (int v = 0; v < 3; ++v) net->fold_dev.fold[v] = F.acc[v];
  CU(cudaStreamCreateWithFlags(&net->stream2, cudaStreamNonBlocking));
  CU(cudaEventCreateWithFlags(&net->ev_n, cudaEventDisableTiming));
  CU(cudaEventCreateWithFlags(&net->ev_d[0], cudaEventDisableTiming));
  CU(cudaEventCreateWithFlags(&net->ev_d[1], cudaEventDisableTiming));
  net->two_launch_ok = true;
  net->two_launch = (flags & (B2B_NET_TWO_LAUNCH | B2B_NET_ONE_LAUNCH)) ||
                    pop.n <= kAutoTwoLaunchMaxNeurons;
  net->one_launch_ok = one_launch_supported(pop, F);
  // delivering CTAs of the one-launch step: 1.5 per SM (in CTAs of kBlock threads) still fit
  // beside the update's in one wave for the populations this form is built for
  net->one_launch_grid = 3 * sms / 2;
  net->one_launch = net->one_launch_ok && (flags & B2B_NET_ONE_LAUNCH);
  return B2B_OK;
}

// ---------------------------------------------------------------------------------------
// Records profiling event `which` (0 before, 1 after) of launch site `site` of step k on s,
// when b2b_profile_graph has set the net's event table; under stream capture the record is
// an event-record node of the graph (an external event), so the replayed graph times the
// launch in its own schedule.
cudaError_t prof_mark(b2b_net* net, int k, int site, int which, cudaStream_t s) {
  if (!net->prof_ev) return cudaSuccess;
  return cudaEventRecordWithFlags(net->prof_ev[((size_t)k * net->prof_sites + site) * 2 + which],
                                  s, cudaEventRecordExternal);
}

b2b_status enqueue_steps(b2b_net* net, int kk) {
  if (net->small) {
    const Pop& pop = net->pops[0];
    CU(prof_mark(net, 0, 0, 0, net->stream));
    CU(launch_small(net->sdev, pop.kind, pop.dtype, net->d_clock, kk, net->cfg.dt,
                    net->d_status, net->stream));
    CU(prof_mark(net, 0, 0, 1, net->stream));
    CU(launch_tick(net->d_clock, kk, net->stream));
    net->launches += 2;
    return B2B_OK;
  }
  if (net->two_launch && net->one_launch) {
    // The same two halves as one grid per step (neuron.cu): consecutive launches on the
    // net's stream order step k+1 after both halves of step k.  Profiling site 0.
    const Pop& pop = net->pops[0];
    cudaStream_t s = net->stream;
    for (int k = 0; k < kk; ++k) {
      CU(prof_mark(net, k, 0, 0, s));
      // the first step of a chunk follows other kernels (the previous chunk's fold and
      // clock tick): an ordinary launch
      CU(launch_one_launch_step(pop, net->fold_dev, net->pdev, net->one_launch_grid,
                                net->one_launch_chained && k > 0, net->d_clock, k, net->cfg.dt,
                                net->d_status, s));
      CU(prof_mark(net, k, 0, 1, s));
      ++net->launches;
    }
    CU(launch_fold_pending(net->pdev, pop.dtype, net->d_clock, kk - 1, s));
    CU(launch_tick(net->d_clock, kk, s));
    net->launches += 2;
    return B2B_OK;
  }
  if (net->two_launch) {
    // Step k's delivery (spikes of steps <= k-1 into acc[k & 1]) and step k's neuron update
    // (which folds in acc[(k-1) & 1]) are independent: the delivery of step k waits for the
    // update of step k-1, the update of step k for the update and the delivery of step k-1.
    // The deliveries run on the second stream; under stream capture this is a graph with
    // two branches per step.  Profiling sites: 0 the delivery, 1 the update.
    const Pop& pop = net->pops[0];
    cudaStream_t s = net->stream, s2 = net->stream2;
    CU(cudaEventRecord(net->ev_n, s));
    for (int k = 0; k < kk; ++k) {
      CU(cudaStreamWaitEvent(s2, net->ev_n, 0));
      CU(prof_mark(net, k, 0, 0, s2));
      CU(launch_pending_delivery(net->pdev, pop.dtype, net->pending_grid, net->d_clock, k, s2));
      CU(prof_mark(net, k, 0, 1, s2));
      CU(cudaEventRecord(net->ev_d[k & 1], s2));
      if (k > 0) CU(cudaStreamWaitEvent(s, net->ev_d[(k - 1) & 1], 0));
      CU(prof_mark(net, k, 1, 0, s));
      CU(launch_pop_step_dev(pop, net->fold_dev, net->d_clock, k, net->cfg.dt, net->d_status,
                             s));
      CU(prof_mark(net, k, 1, 1, s));
      CU(cudaEventRecord(net->ev_n, s));
      net->launches += 2;
    }
    CU(cudaStreamWaitEvent(s, net->ev_d[(kk - 1) & 1], 0));
    CU(launch_fold_pending(net->pdev, pop.dtype, net->d_clock, kk - 1, s));
    CU(launch_tick(net->d_clock, kk, s));
    net->launches += 2;
    return B2B_OK;
  }
  cudaStream_t s = net->stream;
  for (int k = 0; k < kk; ++k) {
    int si = 0;   // profiling site, in the order of b2b_profile's site list
    if (!net->smons.empty()) {
      CU(prof_mark(net, k, si, 0, s));
      CU(launch_statemon(net->d_smons, (int)net->smons.size(), net->smon_max_idx, net->d_clock,
                         k, net->d_status, s));
      CU(prof_mark(net, k, si++, 1, s));
      ++net->launches;
    }
    // the populations' updates of a step are independent: the first on the net's stream,
    // the others side by side on their own streams, joined before the deliveries
    const size_t np = net->pops.size();
    const bool fork = np > 1 && net->pop_streams.size() + 1 == np;
    if (fork) {
      CU(cudaEventRecord(net->ev_pop_fork, s));
      for (cudaStream_t ps : net->pop_streams) CU(cudaStreamWaitEvent(ps, net->ev_pop_fork, 0));
    }
    for (size_t p = 0; p < np; ++p) {
      cudaStream_t ps = fork && p > 0 ? net->pop_streams[p - 1] : s;
      CU(prof_mark(net, k, si, 0, ps));
      CU(launch_pop_step(net->pops[p], net->d_clock, k, net->cfg.dt, net->d_status, ps));
      CU(prof_mark(net, k, si++, 1, ps));
      ++net->launches;
    }
    if (fork)
      for (size_t p = 1; p < np; ++p) {
        CU(cudaEventRecord(net->ev_pop_join[p - 1], net->pop_streams[p - 1]));
        CU(cudaStreamWaitEvent(s, net->ev_pop_join[p - 1], 0));
      }
    for (size_t b = 0; b < net->add_batches.size(); ++b) {
      const auto& B = net->add_batches[b];
      CU(prof_mark(net, k, si, 0, s));
      CU(launch_proj_add_batch(B.data(), (int)B.size(), net->d_clock, k, s,
                               b < net->add_tune.size() ? &net->add_tune[b] : nullptr));
      CU(prof_mark(net, k, si++, 1, s));
      ++net->launches;
    }
    for (const Proj& pr : net->projs) {
      if (pr.effect != B2B_EFFECT_STDP) continue;
      CU(prof_mark(net, k, si, 0, s));
      CU(launch_proj_pre(pr, net->d_clock, k, net->cfg.dt, net->d_status, s));
      CU(prof_mark(net, k, si++, 1, s));
      ++net->launches;
    }
    for (const Proj& pr : net->projs) {
      if (pr.effect != B2B_EFFECT_STDP) continue;
      CU(prof_mark(net, k, si, 0, s));
      CU(launch_proj_post(pr, net->d_clock, k, net->cfg.dt, net->d_status, s));
      CU(prof_mark(net, k, si++, 1, s));
      ++net->launches;
    }
    for (const Pop& pop : net->pops) {
      if (!pop.late_reset) continue;
      CU(prof_mark(net, k, si, 0, s));
      CU(launch_pop_late_reset(pop, net->d_clock, k, s));
      CU(prof_mark(net, k, si++, 1, s));
      ++net->launches;
    }
    if (!net->rmons.empty()) {
      CU(prof_mark(net, k, si, 0, s));
      CU(launch_ratemon(net->d_rmons, (int)net->rmons.size(), net->d_clock, k, net->d_status,
                        s));
      CU(prof_mark(net, k, si++, 1, s));
      ++net->launches;
    }
  }
  CU(launch_tick(net->d_clock, kk, s));
  ++net->launches;
  return B2B_OK;
}

b2b_status refill_rng(b2b_net* net, int kk) {
  for (Pop& pop : net->pops) {
    const int64_t n_uni = pop.kind == KIND_POISSON ? 1
                          : (pop.kind == KIND_MODEL ? pop.minfo.n_uniform : 0);
    const int64_t n_nrm = pop.kind == KIND_MODEL ? pop.minfo.n_normal : 0;
    if (n_uni > 0) {
      const size_t n = (size_t)kk * n_uni * pop.n;
      curandStatus_t st = pop.dtype == B2B_F32
                              ? curandGenerateUniform(net->gen, (float*)pop.rng_buf, n)
                              : curandGenerateUniformDouble(net->gen, (double*)pop.rng_buf, n);
      if (st != CURAND_STATUS_SUCCESS)
        return fail(net, B2B_ERR_CUDA, "curandGenerateUniform failed (%d)", (int)st);
      net->rng_offset += n;
    }
    if (n_nrm > 0) {
      // standard normal numbers for the model's noise terms (xi) and randn(): the buffer
      // brian2cuda refills with curandGenerateNormal (brian2cuda/device.py:751-775); the
      // count is even (populations are padded to 128 neurons), as the generator requires
      const size_t n = (size_t)kk * n_nrm * pop.n;
      curandStatus_t st =
          pop.dtype == B2B_F32
              ? curandGenerateNormal(net->gen, (float*)pop.rng_normal_buf, n, 0.0f, 1.0f)
              : curandGenerateNormalDouble(net->gen, (double*)pop.rng_normal_buf, n, 0.0, 1.0);
      if (st != CURAND_STATUS_SUCCESS)
        return fail(net, B2B_ERR_CUDA, "curandGenerateNormal failed (%d)", (int)st);
      net->rng_offset += n;
    }
  }
  return B2B_OK;
}

// Every device array that holds dynamic state, with its size in bytes.
std::vector<std::pair<void*, size_t>> state_arrays(b2b_net* net) {
  std::vector<std::pair<void*, size_t>> out;
  for (Pop& pop : net->pops) {
    for (int v = 0; v < kMaxVars; ++v)
      if (pop.dev.var[v]) out.emplace_back(pop.dev.var[v], var_size(pop.dtype, v) * pop.n);
    out.emplace_back(pop.dev.ring_idx, sizeof(int32_t) * (size_t)pop.dev.ring_len * pop.n);
    out.emplace_back(pop.dev.ring_cnt, sizeof(int32_t) * (size_t)pop.dev.ring_len);
  }
  for (Proj& pr : net->projs) {
    if (pr.effect != B2B_EFFECT_STDP) continue;
    out.emplace_back(pr.dev.syn4, 4 * real_size(pr.dtype) * pr.n_syn);
  }
  return out;
}

b2b_status capture_graph(b2b_net* net) {
  const int64_t before = net->launches;
  CU(cudaStreamBeginCapture(net->stream, cudaStreamCaptureModeThreadLocal));
  b2b_status st = enqueue_steps(net, net->cfg.steps_per_graph);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(net->stream, &g);
  net->launches = before;
  if (st != B2B_OK) { if (g) cudaGraphDestroy(g); return st; }
  if (e != cudaSuccess) return fail(net, B2B_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
  size_t nodes = 0;
  cudaGraphGetNodes(g, nullptr, &nodes);
  e = cudaGraphInstantiate(&net->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(net, B2B_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
  net->graph_nodes = (int64_t)nodes;
  net->graph_steps = net->cfg.steps_per_graph;
  return B2B_OK;
}

// ---- delays changed between runs -----------------------------------------------------------
// Re-derives the two-launch step's device view from the projections (after a delay change
// added or dropped one); turns the form off when the projections no longer allow it (a delay
// of 0, more projections than one launch takes).  Between runs the pending input is folded
// in, so the per-step form can take over at any run boundary.
void refresh_two_launch(b2b_net* net) {
  if (!net->two_launch_ok) return;
  PendingDev& F = net->pdev;
  bool ok = net->projs.size() <= (size_t)kMaxProjBatch;
  int32_t nd_max = 1;
  for (const Proj& pr : net->projs) {
    ok = ok && pr.effect == B2B_EFFECT_ADD && pr.dmin >= 1;
    for (int m : pr.members) ok = ok && F.acc[net->syns[m].target_var] != nullptr;
    nd_max = std::max(nd_max, pr.dev.nd);
  }
  if (!ok) {
    net->two_launch = false;
    net->two_launch_ok = false;
    net->one_launch = false;
    net->one_launch_ok = false;
    return;
  }
  const Pop& pop = net->pops[0];
  F.pop = pop.dev;
  F.n_proj = (int32_t)net->projs.size();
  F.nd_max = nd_max;
  for (size_t p = 0; p < net->projs.size(); ++p) {
    const Proj& pr = net->projs[p];
    F.proj[p] = pr.dev;
    for (int m : pr.members) {
      const int v = net->syns[m].target_var;
      F.proj[p].targets[v] = F.acc[v];
    }
    F.proj[p].target = F.acc[pr.target_var];
  }
  net->fold_dev = pop.dev;
  for (int v = 0; v < 3; ++v) net->fold_dev.fold[v] = F.acc[v];
  net->one_launch_ok = one_launch_supported(pop, F);
  if (!net->one_launch_ok) net->one_launch = false;
}

// Grows population pi's spike-history ring to new_len slots, keeping the spikes of the last
// old_len - 1 steps (those a delivery can still reach) at their slots in the new ring, and
// points every view of the ring at the new one.  Snapshots hold rings of the old length and
// become unusable.
b2b_status grow_ring(b2b_net* net, int pi, int32_t new_len) {
  Pop& pop = net->pops[pi];
  PopDev& D = pop.dev;
  const int32_t old_len = D.ring_len;
  int32_t* idx = nullptr;
  int32_t* cnt = nullptr;
  CU(dalloc(pop, &idx, (size_t)new_len * pop.n));
  CU(dalloc(pop, &cnt, (size_t)new_len));
  CU(cudaMemset(cnt, 0, sizeof(int32_t) * new_len));
  const int64_t T = net->ts;
  for (int64_t s = T - 1; s >= 0 && s > T - old_len; --s) {
    const int64_t so = s % old_len, sn = s % new_len;
    CU(cudaMemcpy(idx + sn * pop.n, D.ring_idx + so * pop.n, sizeof(int32_t) * pop.n,
                  cudaMemcpyDeviceToDevice));
    CU(cudaMemcpy(cnt + sn, D.ring_cnt + so, sizeof(int32_t), cudaMemcpyDeviceToDevice));
  }
  for (void* old : {(void*)D.ring_idx, (void*)D.ring_cnt}) {
    pop.allocs.erase(std::remove(pop.allocs.begin(), pop.allocs.end(), old), pop.allocs.end());
    cudaFree(old);
  }
  D.ring_idx = idx;
  D.ring_cnt = cnt;
  D.ring_len = new_len;
  pop.max_delay = new_len - 2;
  for (Proj& pr : net->projs) {
    if (pr.src_pop == pi) {
      pr.dev.src_ring_idx = idx;
      pr.dev.src_ring_cnt = cnt;
      pr.dev.src_ring_len = new_len;
    }
    if (pr.effect == B2B_EFFECT_STDP && pr.dst_pop == pi) {
      pr.dev.post_ring_idx = idx;
      pr.dev.post_ring_cnt = cnt;
      pr.dev.post_ring_len = new_len;
    }
  }
  if (!net->rmons.empty()) {
    std::vector<RateMonDev> devs;
    for (RateMon& m : net->rmons) {
      if (net->groups[m.gid].pop == pi) {
        m.dev.ring_idx = idx;
        m.dev.ring_cnt = cnt;
        m.dev.ring_len = new_len;
      }
      devs.push_back(m.dev);
    }
    CU(cudaMemcpy(net->d_rmons, devs.data(), sizeof(RateMonDev) * devs.size(),
                  cudaMemcpyHostToDevice));
  }
  for (Snapshot& sn : net->snapshots) sn.valid = false;
  return B2B_OK;
}

// Drops the retired projections whose last spikes have arrived.
b2b_status drop_retired(b2b_net* net) {
  bool any = false;
  for (size_t p = 0; p < net->projs.size();) {
    Proj& pr = net->projs[p];
    if (pr.retire_after >= 0 && net->ts > pr.retire_after) {
      for (void* a : pr.allocs) cudaFree(a);
      net->projs.erase(net->projs.begin() + p);
      any = true;
    } else {
      ++p;
    }
  }
  if (any) {
    build_add_batches(net);
    refresh_two_launch(net);
    if (net->graph) {
      cudaGraphExecDestroy(net->graph);
      net->graph = nullptr;
    }
  }
  return B2B_OK;
}

// Copies the random numbers the last chunk drew for group gid to the host: a Poisson group's
// uniforms (n = group size per step), or a generated model's uniforms / normals (n = draws
// per step x group size, draw-major).
b2b_status rng_buffer_get(b2b_net* net, int32_t gid, bool normal, void* host, int64_t steps,
                          int64_t n) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(gid >= 0 && gid < (int)net->groups.size(), B2B_ERR_INVALID_ARG, "bad group %d", gid);
  const Group& g = net->groups[gid];
  int64_t draws = 0;
  if (g.kind == KIND_POISSON && !normal) draws = 1;
  if (g.kind == KIND_MODEL) draws = normal ? g.minfo.n_normal : g.minfo.n_uniform;
  CHECK(draws > 0, B2B_ERR_INVALID_ARG, "group %d draws no %s numbers", gid,
        normal ? "normal" : "uniform");
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  CHECK(host && n == draws * g.n && steps > 0 && steps <= net->last_chunk_steps,
        B2B_ERR_INVALID_ARG, "bad shape");
  const Pop& pop = net->pops[g.pop];
  const uint8_t* buf = static_cast<const uint8_t*>(normal ? pop.rng_normal_buf : pop.rng_buf);
  const size_t rs = real_size(pop.dtype);
  CU(cudaStreamSynchronize(net->stream));
  for (int64_t k = 0; k < steps; ++k)
    for (int64_t d = 0; d < draws; ++d)
      CU(cudaMemcpy((uint8_t*)host + rs * (k * n + d * g.n),
                    buf + rs * ((k * draws + d) * pop.n + g.offset), rs * g.n,
                    cudaMemcpyDeviceToHost));
  return B2B_OK;
}

// Launch sites of one step, in the order enqueue_steps marks them for profiling: the state
// monitors (kind 9), each population (1), each additive delivery launch (6), each STDP
// projection's on_pre (2) and on_post (3), each deferred reset (4), the rate monitors (10);
// the two-launch step: its delivery (5) and update (1); the one-launch step: its kernel (13);
// the one-CTA small path: its kernel (7).
struct ProfSite { int kind; int idx; };
std::vector<ProfSite> profile_sites(const b2b_net* net) {
  std::vector<ProfSite> sites;
  if (net->small) {
    sites.push_back({7, 0});
  } else if (net->two_launch && net->one_launch) {
    sites.push_back({13, 0});
  } else if (net->two_launch) {
    sites.push_back({5, 0});
    sites.push_back({1, 0});
  } else {
    if (!net->smons.empty()) sites.push_back({9, 0});
    for (size_t p = 0; p < net->pops.size(); ++p) sites.push_back({1, (int)p});
    for (size_t b = 0; b < net->add_batches.size(); ++b) sites.push_back({6, (int)b});
    for (size_t p = 0; p < net->projs.size(); ++p)
      if (net->projs[p].effect == B2B_EFFECT_STDP) sites.push_back({2, (int)p});
    for (size_t p = 0; p < net->projs.size(); ++p)
      if (net->projs[p].effect == B2B_EFFECT_STDP) sites.push_back({3, (int)p});
    for (size_t p = 0; p < net->pops.size(); ++p)
      if (net->pops[p].late_reset) sites.push_back({4, (int)p});
    if (!net->rmons.empty()) sites.push_back({10, 0});
  }
  return sites;
}

}  // namespace

// =========================================================================================
extern "C" {

int32_t b2b_abi_version(void) { return B2B_ABI_VERSION; }

const char* b2b_status_string(b2b_status s) {
  switch (s) {
    case B2B_OK: return "ok";
    case B2B_ERR_INVALID_ARG: return "invalid argument";
    case B2B_ERR_OOM: return "out of memory";
    case B2B_ERR_QUEUE_OVERFLOW: return "device buffer overflow";
    case B2B_ERR_TIMEOUT: return "device wait timed out";
    case B2B_ERR_CUDA: return "CUDA error";
    case B2B_ERR_STATE: return "invalid state";
    case B2B_ERR_UNSUPPORTED: return "unsupported";
    case B2B_ERR_INDEX: return "index out of range";
    default: return "unknown status";
  }
}

b2b_status b2b_last_error(const b2b_net* net, char* buf, size_t len) {
  if (!net || !buf || len == 0) return B2B_ERR_INVALID_ARG;
  std::snprintf(buf, len, "%s", net->err.c_str());
  return B2B_OK;
}

b2b_status b2b_create(const b2b_config* cfg, b2b_net** out) {
  if (!cfg || !out) return B2B_ERR_INVALID_ARG;
  if (!(cfg->dt > 0) || !std::isfinite(cfg->dt)) return B2B_ERR_INVALID_ARG;
  *out = nullptr;
  b2b_net* net = new (std::nothrow) b2b_net();
  if (!net) return B2B_ERR_OOM;
  net->cfg = *cfg;
  if (net->cfg.steps_per_graph <= 0) net->cfg.steps_per_graph = 50;
  cudaError_t e = cudaSetDevice(cfg->device);
  if (e == cudaSuccess) {
    if (cfg->stream) {
      net->stream = (cudaStream_t)cfg->stream;
    } else {
      e = cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking);
      net->own_stream = e == cudaSuccess;
    }
  }
  if (e == cudaSuccess) e = cudaMalloc(&net->d_clock, sizeof(int64_t));
  if (e == cudaSuccess) e = cudaMalloc(&net->d_status, sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMemset(net->d_clock, 0, sizeof(int64_t));
  if (e == cudaSuccess) e = cudaMemset(net->d_status, 0, sizeof(int32_t));
  if (e != cudaSuccess) {
    b2b_destroy(net);
    return e == cudaErrorMemoryAllocation ? B2B_ERR_OOM : B2B_ERR_CUDA;
  }
  *out = net;
  return B2B_OK;
}

b2b_status b2b_destroy(b2b_net* net) {
  if (!net) return B2B_ERR_INVALID_ARG;
  cudaSetDevice(net->cfg.device);
  if (net->stream) cudaStreamSynchronize(net->stream);
  const std::vector<b2b_hines*> hines = net->hines;
  for (b2b_hines* h : hines) b2b_hines_destroy(h);
  if (net->graph) cudaGraphExecDestroy(net->graph);
  if (net->gen) curandDestroyGenerator(net->gen);
  for (Pop& p : net->pops)
    for (void* a : p.allocs) cudaFree(a);
  for (Proj& p : net->projs)
    for (void* a : p.allocs) cudaFree(a);
  for (Snapshot& sn : net->snapshots)
    for (void* a : sn.buffers) cudaFree(a);
  for (void* a : net->pending_allocs) cudaFree(a);
  if (net->pull_buf) cudaFree(net->pull_buf);
  if (net->fetch_pinned) cudaFreeHost(net->fetch_pinned);
  if (net->stream2) cudaStreamDestroy(net->stream2);
  for (cudaStream_t ps : net->pop_streams) {
    cudaStreamSynchronize(ps);
    cudaStreamDestroy(ps);
  }
  if (net->ev_pop_fork) cudaEventDestroy(net->ev_pop_fork);
  for (cudaEvent_t ev : net->ev_pop_join)
    if (ev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : {net->ev_n, net->ev_d[0], net->ev_d[1]})
    if (ev) cudaEventDestroy(ev);
  for (void* a : net->mon_allocs) cudaFree(a);
  cudaFree(net->d_clock);
  cudaFree(net->d_status);
  if (net->own_stream) cudaStreamDestroy(net->stream);
  delete net;
  return B2B_OK;
}

b2b_status b2b_group_lif(b2b_net* net, int64_t n, int32_t dtype, const b2b_lif_params* p,
                         int32_t* gid) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(p != nullptr, B2B_ERR_INVALID_ARG, "params is NULL");
  CHECK(!(p->taum <= 0) && !(p->taue < 0) && !(p->taui < 0) && !(p->refractory < 0),
        B2B_ERR_INVALID_ARG, "time constants must be positive");
  GUARD_BEGIN
  Group g;
  g.kind = KIND_LIF; g.n = n; g.dtype = dtype; g.lif = *p;
  return add_group(net, std::move(g), gid);
  GUARD_END
}

b2b_status b2b_group_hh(b2b_net* net, int64_t n, int32_t dtype, const b2b_hh_params* p,
                        int32_t* gid) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(p != nullptr, B2B_ERR_INVALID_ARG, "params is NULL");
  CHECK(p->Cm > 0 && p->taue > 0 && p->taui > 0 && !(p->refractory < 0), B2B_ERR_INVALID_ARG,
        "Cm and time constants must be positive");
  GUARD_BEGIN
  Group g;
  g.kind = KIND_HH; g.n = n; g.dtype = dtype; g.hh = *p;
  return add_group(net, std::move(g), gid);
  GUARD_END
}

b2b_status b2b_group_hh_surrogate(b2b_net* net, int32_t gid, b2b_mlp* m, double tol,
                                  int32_t judge) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(!net->finalized, B2B_ERR_STATE, "attach the surrogate before b2b_finalize");
  CHECK(gid >= 0 && gid < (int32_t)net->groups.size(), B2B_ERR_INVALID_ARG, "bad group id");
  CHECK(m != nullptr && tol >= 0 && std::isfinite(tol) && (judge == 0 || judge == 1),
        B2B_ERR_INVALID_ARG, "bad surrogate arguments");
  Group& g0 = net->groups[gid];
  CHECK(g0.kind == KIND_HH && g0.dtype == B2B_F32, B2B_ERR_UNSUPPORTED,
        "the gating surrogate applies to float32 HH groups");
  for (Group& g : net->groups) {
    if (g.kind != KIND_HH || g.dtype != B2B_F32) continue;
    g.surr = m;
    g.surr_tol = tol;
    g.surr_judge = judge;
  }
  return B2B_OK;
}

b2b_status b2b_surrogate_stats(b2b_net* net, int32_t gid, int64_t* updates, int64_t* fallbacks) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  CHECK(gid >= 0 && gid < (int32_t)net->groups.size() && updates && fallbacks,
        B2B_ERR_INVALID_ARG, "bad arguments");
  const Pop& pop = net->pops[net->groups[gid].pop];
  CHECK(pop.surr_cnt != nullptr, B2B_ERR_STATE, "no surrogate attached to this group");
  unsigned long long c[2] = {0, 0};
  CU(cudaMemcpyAsync(c, pop.surr_cnt, sizeof c, cudaMemcpyDeviceToHost, net->stream));
  CU(cudaStreamSynchronize(net->stream));
  *updates = (int64_t)c[0];
  *fallbacks = (int64_t)c[1];
  return B2B_OK;
}

b2b_status b2b_hh_gating_sample(b2b_net* net, int32_t gid, float* dev_x, int64_t n) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  CHECK(gid >= 0 && gid < (int32_t)net->groups.size() && dev_x != nullptr, B2B_ERR_INVALID_ARG,
        "bad arguments");
  CHECK((reinterpret_cast<uintptr_t>(dev_x) & 15) == 0, B2B_ERR_INVALID_ARG,
        "dev_x must be 16-byte aligned");
  const Group& g = net->groups[gid];
  CHECK(g.kind == KIND_HH && g.dtype == B2B_F32, B2B_ERR_UNSUPPORTED,
        "sampling applies to float32 HH groups");
  CHECK(n >= 0 && n <= g.n, B2B_ERR_INVALID_ARG, "n exceeds the group size");
  if (n == 0) return B2B_OK;
  CU(launch_hh_sample(net->pops[g.pop], g.offset, n, dev_x, net->stream));
  return B2B_OK;
}

b2b_status b2b_group_poisson(b2b_net* net, int64_t n, int32_t dtype, double rate_hz,
                             int32_t* gid) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(rate_hz >= 0 && std::isfinite(rate_hz), B2B_ERR_INVALID_ARG, "bad rate");
  GUARD_BEGIN
  Group g;
  g.kind = KIND_POISSON; g.n = n; g.dtype = dtype; g.rate = rate_hz;
  return add_group(net, std::move(g), gid);
  GUARD_END
}

b2b_status b2b_group_spikegen(b2b_net* net, int64_t n, int64_t n_spikes, const int32_t* idx,
                              const int64_t* step, int32_t* gid) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(n_spikes >= 0 && (n_spikes == 0 || (idx && step)), B2B_ERR_INVALID_ARG,
        "bad spike list");
  GUARD_BEGIN
  Group g;
  g.kind = KIND_SPIKEGEN; g.n = n; g.dtype = B2B_F32;
  std::vector<std::pair<int64_t, int32_t>> ent;
  for (int64_t k = 0; k < n_spikes; ++k) {
    CHECK(idx[k] >= 0 && idx[k] < n && step[k] >= 0, B2B_ERR_INDEX,
          "spike %lld: index %d / step %lld out of range", (long long)k, idx[k],
          (long long)step[k]);
    ent.emplace_back(step[k], idx[k]);
  }
  std::sort(ent.begin(), ent.end());
  for (size_t k = 1; k < ent.size(); ++k)
    CHECK(ent[k] != ent[k - 1], B2B_ERR_INVALID_ARG, "neuron %d spikes twice in step %lld",
          ent[k].second, (long long)ent[k].first);
  for (auto& e : ent) { g.sg_step.push_back(e.first); g.sg_idx.push_back(e.second); }
  return add_group(net, std::move(g), gid);
  GUARD_END
}

b2b_status b2b_poisson_input(b2b_net* net, int32_t gid, int32_t var, int64_t n_inputs,
                             double rate_hz, double weight, int32_t* pid) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(!net->finalized, B2B_ERR_STATE, "PoissonInputs must be added before b2b_finalize");
  CHECK(gid >= 0 && gid < (int)net->groups.size(), B2B_ERR_INVALID_ARG, "bad group %d", gid);
  Group& g = net->groups[gid];
  CHECK(g.kind == KIND_LIF || g.kind == KIND_HH, B2B_ERR_INVALID_ARG,
        "a PoissonInput targets a LIF or HH group");
  CHECK(var == B2B_VAR_V || var == B2B_VAR_GE || var == B2B_VAR_GI, B2B_ERR_INVALID_ARG,
        "a PoissonInput targets v, ge or gi");
  CHECK((int)g.pins.size() < kMaxPoissonInputs, B2B_ERR_UNSUPPORTED,
        "at most %d PoissonInputs per group", kMaxPoissonInputs);
  const double p = rate_hz * net->cfg.dt;
  CHECK(n_inputs >= 0 && std::isfinite(p) && p >= 0 && p <= 1 && std::isfinite(weight),
        B2B_ERR_INVALID_ARG, "bad PoissonInput (N %lld, rate*dt %g)", (long long)n_inputs, p);
  GUARD_BEGIN
  PoissonIn in{};
  in.n = n_inputs;
  in.reverse = p > 0.5 ? 1 : 0;
  const double pp = in.reverse ? 1.0 - p : p;
  const double q = 1.0 - pp;
  in.qn = std::pow(q, (double)n_inputs);
  in.s = q > 0 ? pp / q : 0.0;
  in.a = (double)(n_inputs + 1) * in.s;
  in.weight = weight;
  in.var = var;
  in.id = (uint32_t)net->n_pins;
  in.k0 = (uint32_t)net->cfg.seed;
  in.k1 = (uint32_t)(net->cfg.seed >> 32) ^ 0xB1A0u;
  g.pins.push_back(in);
  if (pid) *pid = net->n_pins;
  ++net->n_pins;
  return B2B_OK;
  GUARD_END
}

b2b_status b2b_timedarray(b2b_net* net, int32_t gid, const double* values, int64_t rows,
                          int64_t cols, double dt_array) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(!net->finalized, B2B_ERR_STATE, "TimedArrays must be set before b2b_finalize");
  CHECK(gid >= 0 && gid < (int)net->groups.size(), B2B_ERR_INVALID_ARG, "bad group %d", gid);
  Group& g = net->groups[gid];
  CHECK(g.kind == KIND_LIF || g.kind == KIND_HH || g.kind == KIND_POISSON, B2B_ERR_INVALID_ARG,
        "a TimedArray drives a LIF, HH or Poisson group");
  CHECK(values && rows > 0 && (cols == 1 || cols == g.n), B2B_ERR_INVALID_ARG,
        "values must be [rows >= 1][1 or the group's %lld neurons]", (long long)g.n);
  CHECK(std::isfinite(dt_array) && dt_array > 0, B2B_ERR_INVALID_ARG, "bad dt_array");
  // aligned time grids: dt_array = m dt (row = ts / m) or dt = r dt_array (row = ts * r)
  const double dt = net->cfg.dt;
  int64_t mul = 1, div = 1;
  if (dt_array >= dt) {
    div = std::llround(dt_array / dt);
    CHECK(std::fabs(dt_array / dt - (double)div) <= 1e-6, B2B_ERR_INVALID_ARG,
          "dt_array %g is not a multiple of dt %g", dt_array, dt);
  } else {
    mul = std::llround(dt / dt_array);
    CHECK(std::fabs(dt / dt_array - (double)mul) <= 1e-6, B2B_ERR_INVALID_ARG,
          "dt %g is not a multiple of dt_array %g", dt, dt_array);
  }
  GUARD_BEGIN
  g.ta.assign(values, values + rows * cols);
  g.ta_rows = rows;
  g.ta_cols = cols;
  g.ta_mul = mul;
  g.ta_div = div;
  return B2B_OK;
  GUARD_END
}

b2b_status b2b_spikegen_period(b2b_net* net, int32_t gid, int64_t period_steps) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(!net->finalized, B2B_ERR_STATE, "the period must be set before b2b_finalize");
  CHECK(gid >= 0 && gid < (int)net->groups.size() &&
            net->groups[gid].kind == KIND_SPIKEGEN,
        B2B_ERR_INVALID_ARG, "group %d is not a SpikeGeneratorGroup", gid);
  Group& g = net->groups[gid];
  CHECK(period_steps >= 0, B2B_ERR_INVALID_ARG, "negative period");
  for (int64_t s : g.sg_step)
    CHECK(period_steps == 0 || s < period_steps, B2B_ERR_INVALID_ARG,
          "spike at step %lld is not inside the period of %lld steps", (long long)s,
          (long long)period_steps);
  g.sg_period = period_steps;
  return B2B_OK;
}

b2b_status b2b_state_set(b2b_net* net, int32_t gid, int32_t var, const void* host, int64_t n) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(gid >= 0 && gid < (int)net->groups.size(), B2B_ERR_INVALID_ARG, "bad group %d", gid);
  Group& g = net->groups[gid];
  CHECK(kind_has_var(g.kind, var, g.minfo.n_vars), B2B_ERR_INVALID_ARG,
        "group %d has no variable %d", gid, var);
  CHECK(host && n == g.n, B2B_ERR_INVALID_ARG, "expected %lld values", (long long)g.n);
  const size_t es = var_size(g.dtype, var);
  GUARD_BEGIN
  if (!net->finalized) {
    g.staged[var].assign((const uint8_t*)host, (const uint8_t*)host + es * n);
    return B2B_OK;
  }
  uint8_t* d = (uint8_t*)net->pops[g.pop].dev.var[var] + es * g.offset;
  CU(cudaMemcpyAsync(d, host, es * n, cudaMemcpyHostToDevice, net->stream));
  CU(cudaStreamSynchronize(net->stream));
  return B2B_OK;
  GUARD_END
}

b2b_status b2b_state_get(b2b_net* net, int32_t gid, int32_t var, void* host, int64_t n) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(gid >= 0 && gid < (int)net->groups.size(), B2B_ERR_INVALID_ARG, "bad group %d", gid);
  Group& g = net->groups[gid];
  CHECK(kind_has_var(g.kind, var, g.minfo.n_vars), B2B_ERR_INVALID_ARG,
        "group %d has no variable %d", gid, var);
  CHECK(host && n == g.n, B2B_ERR_INVALID_ARG, "expected %lld values", (long long)g.n);
  CHECK(net->finalized, B2B_ERR_STATE, "state is on the device only after b2b_finalize");
  const size_t es = var_size(g.dtype, var);
  const uint8_t* d = (const uint8_t*)net->pops[g.pop].dev.var[var] + es * g.offset;
  CU(cudaMemcpyAsync(host, d, es * n, cudaMemcpyDeviceToHost, net->stream));
  CU(cudaStreamSynchronize(net->stream));
  return B2B_OK;
}

b2b_status b2b_state_ptr(b2b_net* net, int32_t gid, int32_t var, void** dev, int64_t* n) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(gid >= 0 && gid < (int)net->groups.size(), B2B_ERR_INVALID_ARG, "bad group %d", gid);
  Group& g = net->groups[gid];
  CHECK(kind_has_var(g.kind, var, g.minfo.n_vars), B2B_ERR_INVALID_ARG,
        "group %d has no variable %d", gid, var);
  CHECK(dev && n, B2B_ERR_INVALID_ARG, "NULL output");
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  *dev = (uint8_t*)net->pops[g.pop].dev.var[var] + var_size(g.dtype, var) * g.offset;
  *n = g.n;
  return B2B_OK;
}

b2b_status b2b_synapses(b2b_net* net, int32_t pre_gid, int32_t post_gid, int32_t target_var,
                        int32_t effect, int64_t n_syn, const int32_t* i, const int32_t* j,
                        const void* w, double w_scalar, const int32_t* delay_steps,
                        int32_t delay_scalar, const b2b_stdp_params* stdp, int32_t* sid) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(pre_gid >= 0 && pre_gid < (int)net->groups.size() && post_gid >= 0 &&
            post_gid < (int)net->groups.size(),
        B2B_ERR_INVALID_ARG, "bad group id");
  CHECK(n_syn >= 0 && (n_syn == 0 || (i && j)), B2B_ERR_INVALID_ARG, "bad synapse arrays");
  CHECK(effect != B2B_EFFECT_STDP || stdp, B2B_ERR_INVALID_ARG, "STDP needs parameters");
  CHECK(delay_steps || delay_scalar >= 0, B2B_ERR_INVALID_ARG, "negative delay");
  GUARD_BEGIN
  const Group& gpre = net->groups[pre_gid];
  const Group& gpost = net->groups[post_gid];
  Syn s;
  s.pre_gid = pre_gid; s.post_gid = post_gid; s.target_var = target_var; s.effect = effect;
  s.n = n_syn;
  s.i.assign(i, i + n_syn);
  s.j.assign(j, j + n_syn);
  int32_t dmin = delay_scalar, dmax = delay_scalar;
  for (int64_t k = 0; k < n_syn; ++k) {
    CHECK(i[k] >= 0 && i[k] < gpre.n && j[k] >= 0 && j[k] < gpost.n, B2B_ERR_INDEX,
          "synapse %lld: (%d, %d) outside (%lld, %lld)", (long long)k, i[k], j[k],
          (long long)gpre.n, (long long)gpost.n);
  }
  if (delay_steps) {
    s.delay.assign(delay_steps, delay_steps + n_syn);
    dmin = n_syn ? INT32_MAX : 0;
    dmax = 0;
    for (int64_t k = 0; k < n_syn; ++k) {
      CHECK(delay_steps[k] >= 0, B2B_ERR_INVALID_ARG, "negative delay at synapse %lld",
            (long long)k);
      dmin = std::min(dmin, delay_steps[k]);
      dmax = std::max(dmax, delay_steps[k]);
    }
  }
  s.delay_scalar = delay_scalar;
  s.dmin = dmin; s.dmax = dmax;
  s.pre_lo = 0;
  s.pre_hi = (int32_t)gpre.n;
  if (w) {
    const size_t rs = real_size(gpost.dtype);
    s.w.assign((const uint8_t*)w, (const uint8_t*)w + rs * n_syn);
  }
  s.w_scalar = w_scalar;
  if (stdp) s.stdp = *stdp;
  return add_syn(net, std::move(s), sid);
  GUARD_END
}

b2b_status b2b_synapses_random(b2b_net* net, int32_t pre_gid, int32_t pre_lo, int32_t pre_hi,
                               int32_t post_gid, int32_t target_var, double p, int32_t dmin,
                               int32_t dmax, double w, uint64_t seed, int32_t* sid) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(p >= 0 && p <= 1, B2B_ERR_INVALID_ARG, "p must be in [0, 1]");
  CHECK(dmin >= 0 && dmax >= dmin, B2B_ERR_INVALID_ARG, "bad delay range");
  CHECK(pre_gid >= 0 && pre_gid < (int)net->groups.size(), B2B_ERR_INVALID_ARG,
        "bad pre group %d", pre_gid);
  CHECK(pre_lo >= 0 && pre_lo < pre_hi && pre_hi <= net->groups[pre_gid].n, B2B_ERR_INVALID_ARG,
        "bad presynaptic range [%d, %d)", pre_lo, pre_hi);
  GUARD_BEGIN
  Syn s;
  s.pre_gid = pre_gid; s.post_gid = post_gid; s.target_var = target_var;
  s.effect = B2B_EFFECT_ADD;
  s.generated = true;
  s.p = p; s.gdmin = dmin; s.gdmax = dmax; s.gseed = seed;
  s.dmin = dmin; s.dmax = dmax;
  s.pre_lo = pre_lo;
  s.pre_hi = pre_hi;
  s.w_scalar = w;
  return add_syn(net, std::move(s), sid);
  GUARD_END
}

b2b_status b2b_spikemon(b2b_net* net, int32_t gid, int64_t capacity) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(!net->finalized, B2B_ERR_STATE, "monitors must be added before b2b_finalize");
  CHECK(gid >= 0 && gid < (int)net->groups.size(), B2B_ERR_INVALID_ARG, "bad group %d", gid);
  CHECK(capacity > 0, B2B_ERR_INVALID_ARG, "capacity must be positive");
  net->groups[gid].mon_cap = capacity;
  return B2B_OK;
}

b2b_status b2b_statemon(b2b_net* net, int32_t gid, int32_t var, const int64_t* idx, int64_t n,
                        int32_t every, int64_t capacity, int32_t* mid) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(!net->finalized, B2B_ERR_STATE, "monitors must be added before b2b_finalize");
  CHECK(gid >= 0 && gid < (int)net->groups.size() && mid, B2B_ERR_INVALID_ARG,
        "bad group %d", gid);
  const Group& g = net->groups[gid];
  CHECK(kind_has_var(g.kind, var, g.minfo.n_vars), B2B_ERR_INVALID_ARG,
        "group %d has no variable %d", gid, var);
  CHECK(n >= 0 && (idx || n == 0) && every >= 1 && capacity > 0, B2B_ERR_INVALID_ARG,
        "bad indices, interval or capacity");
  StateMon m;
  m.gid = gid;
  m.var = var;
  m.every = every;
  m.cap = capacity;
  for (int64_t k = 0; k < n; ++k) {
    CHECK(idx[k] >= 0 && idx[k] < g.n, B2B_ERR_INDEX, "index %lld outside group %d",
          (long long)idx[k], gid);
    m.idx.push_back(idx[k]);
  }
  net->smons.push_back(std::move(m));
  *mid = (int32_t)net->smons.size() - 1;
  return B2B_OK;
}

b2b_status b2b_statemon_get(b2b_net* net, int32_t mid, int64_t* n_records, int64_t* steps,
                            void* values, int64_t cap) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  CHECK(mid >= 0 && mid < (int)net->smons.size() && n_records && cap >= 0,
        B2B_ERR_INVALID_ARG, "bad state monitor %d", mid);
  const StateMonDev& D = net->smons[mid].dev;
  CU(cudaStreamSynchronize(net->stream));
  unsigned long long cnt = 0;
  CU(cudaMemcpy(&cnt, D.cnt, sizeof(cnt), cudaMemcpyDeviceToHost));
  *n_records = (int64_t)cnt;
  const int64_t m = std::min<int64_t>((int64_t)cnt, cap);
  if (m > 0 && steps) CU(cudaMemcpy(steps, D.steps, sizeof(int64_t) * m, cudaMemcpyDeviceToHost));
  if (m > 0 && values)
    CU(cudaMemcpy(values, D.buf, (size_t)D.es * (size_t)D.n_idx * (size_t)m,
                  cudaMemcpyDeviceToHost));
  return B2B_OK;
}

b2b_status b2b_ratemon(b2b_net* net, int32_t gid, int64_t capacity, int32_t* mid) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(!net->finalized, B2B_ERR_STATE, "monitors must be added before b2b_finalize");
  CHECK(gid >= 0 && gid < (int)net->groups.size() && mid, B2B_ERR_INVALID_ARG,
        "bad group %d", gid);
  CHECK(capacity > 0, B2B_ERR_INVALID_ARG, "capacity must be positive");
  RateMon m;
  m.gid = gid;
  m.cap = capacity;
  net->rmons.push_back(m);
  *mid = (int32_t)net->rmons.size() - 1;
  return B2B_OK;
}

b2b_status b2b_ratemon_get(b2b_net* net, int32_t mid, int64_t* n_records, int64_t* steps,
                           int32_t* counts, int64_t cap) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  CHECK(mid >= 0 && mid < (int)net->rmons.size() && n_records && cap >= 0,
        B2B_ERR_INVALID_ARG, "bad rate monitor %d", mid);
  const RateMonDev& D = net->rmons[mid].dev;
  CU(cudaStreamSynchronize(net->stream));
  unsigned long long cnt = 0;
  CU(cudaMemcpy(&cnt, D.cnt, sizeof(cnt), cudaMemcpyDeviceToHost));
  *n_records = (int64_t)cnt;
  const int64_t m = std::min<int64_t>((int64_t)cnt, cap);
  if (m > 0 && steps) CU(cudaMemcpy(steps, D.steps, sizeof(int64_t) * m, cudaMemcpyDeviceToHost));
  if (m > 0 && counts) CU(cudaMemcpy(counts, D.buf, sizeof(int32_t) * m, cudaMemcpyDeviceToHost));
  return B2B_OK;
}

b2b_status b2b_finalize(b2b_net* net) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(!net->finalized, B2B_ERR_STATE, "already finalized");
  GUARD_BEGIN
  b2b_status st = finalize_pops(net);
  if (st == B2B_OK) st = finalize_projs(net);
  if (st == B2B_OK) st = setup_monitors(net);
  if (st == B2B_OK) st = setup_two_launch(net);
  if (st == B2B_OK) st = setup_small(net);
  if (st != B2B_OK) return st;
  if (net->pops.size() > 1) {
    CU(cudaEventCreateWithFlags(&net->ev_pop_fork, cudaEventDisableTiming));
    for (size_t p = 1; p < net->pops.size(); ++p) {
      cudaStream_t ps = nullptr;
      cudaEvent_t ev = nullptr;
      CU(cudaStreamCreateWithFlags(&ps, cudaStreamNonBlocking));
      net->pop_streams.push_back(ps);
      CU(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      net->ev_pop_join.push_back(ev);
    }
  }
  CU(cudaMemcpy(net->d_clock, &net->ts, sizeof(int64_t), cudaMemcpyHostToDevice));
  CU(cudaDeviceSynchronize());
  net->finalized = true;
  return B2B_OK;
  GUARD_END
}

b2b_status b2b_run(b2b_net* net, int64_t n_steps) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  CHECK(n_steps >= 0, B2B_ERR_INVALID_ARG, "negative step count");
  const int K = net->cfg.steps_per_graph;
  const bool use_graph = !(net->cfg.flags & B2B_NET_NO_GRAPH);
  if (b2b_status st = drop_retired(net)) return st;
  while (n_steps > 0) {
    const int kk = (int)std::min<int64_t>(n_steps, K);
    if (b2b_status st = refill_rng(net, kk)) return st;
    if (use_graph && kk == K) {
      if (!net->graph) {
        if (b2b_status st = capture_graph(net)) return st;
      }
      CU(cudaGraphLaunch(net->graph, net->stream));
      net->launches += net->graph_nodes;
    } else {
      if (b2b_status st = enqueue_steps(net, kk)) return st;
    }
    net->last_chunk_steps = kk;
    net->ts += kk;
    n_steps -= kk;
  }
  return B2B_OK;
}

b2b_status b2b_profile(b2b_net* net, int64_t n_steps, double* mean_ms, int32_t* site_kind,
                       int32_t cap, int32_t* n_sites) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  CHECK(n_steps > 0 && n_sites, B2B_ERR_INVALID_ARG, "bad arguments");
  GUARD_BEGIN
  using Site = ProfSite;
  const std::vector<Site> sites = profile_sites(net);
  const size_t ns = sites.size();
  std::vector<cudaEvent_t> ev(2 * ns);
  for (auto& e : ev) CU(cudaEventCreate(&e));
  std::vector<double> acc(ns, 0.0);
  b2b_status result = B2B_OK;
  for (int64_t step = 0; step < n_steps && result == B2B_OK; ++step) {
    if ((result = refill_rng(net, 1)) != B2B_OK) break;
    for (size_t k = 0; k < ns && result == B2B_OK; ++k) {
      const Site& s = sites[k];
      cudaEventRecord(ev[2 * k], net->stream);
      cudaError_t e = cudaSuccess;
      const int64_t* clk = net->d_clock;
      if (s.kind == 1)
        e = launch_pop_step_dev(net->pops[s.idx], net->two_launch ? net->fold_dev : net->pops[s.idx].dev,
                                clk, 0, net->cfg.dt, net->d_status, net->stream);
      if (s.kind == 6)
        e = launch_proj_add_batch(net->add_batches[s.idx].data(), (int)net->add_batches[s.idx].size(),
                                  clk, 0, net->stream,
                                  (size_t)s.idx < net->add_tune.size() ? &net->add_tune[s.idx]
                                                                       : nullptr);
      if (s.kind == 2) e = launch_proj_pre(net->projs[s.idx], clk, 0, net->cfg.dt, net->d_status, net->stream);
      if (s.kind == 3) e = launch_proj_post(net->projs[s.idx], clk, 0, net->cfg.dt, net->d_status, net->stream);
      if (s.kind == 4) e = launch_pop_late_reset(net->pops[s.idx], clk, 0, net->stream);
      if (s.kind == 9)
        e = launch_statemon(net->d_smons, (int)net->smons.size(), net->smon_max_idx, clk, 0,
                            net->d_status, net->stream);
      if (s.kind == 10)
        e = launch_ratemon(net->d_rmons, (int)net->rmons.size(), clk, 0, net->d_status,
                           net->stream);
      if (s.kind == 7)
        e = launch_small(net->sdev, net->pops[0].kind, net->pops[0].dtype, clk, 1, net->cfg.dt,
                         net->d_status, net->stream);
      if (s.kind == 5)
        e = launch_pending_delivery(net->pdev, net->pops[0].dtype, net->pending_grid, clk, 0,
                                    net->stream);
      if (s.kind == 13)
        e = launch_one_launch_step(net->pops[0], net->fold_dev, net->pdev, net->one_launch_grid,
                                   false, clk, 0, net->cfg.dt, net->d_status, net->stream);
      cudaEventRecord(ev[2 * k + 1], net->stream);
      if (e != cudaSuccess) result = fail(net, B2B_ERR_CUDA, "profile launch: %s", cudaGetErrorString(e));
      ++net->launches;
    }
    if (result != B2B_OK) break;
    cudaError_t e = launch_tick(net->d_clock, 1, net->stream);
    ++net->launches;
    if (e == cudaSuccess) e = cudaStreamSynchronize(net->stream);
    if (e != cudaSuccess) { result = fail(net, B2B_ERR_CUDA, "profile: %s", cudaGetErrorString(e)); break; }
    for (size_t k = 0; k < ns; ++k) {
      float ms = 0;
      cudaEventElapsedTime(&ms, ev[2 * k], ev[2 * k + 1]);
      acc[k] += ms;
    }
    net->ts += 1;
    net->last_chunk_steps = 1;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (result == B2B_OK && net->two_launch) {
    cudaError_t e = launch_fold_pending(net->pdev, net->pops[0].dtype, net->d_clock, -1, net->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(net->stream);
    if (e != cudaSuccess) result = fail(net, B2B_ERR_CUDA, "profile fold: %s", cudaGetErrorString(e));
  }
  if (result != B2B_OK) return result;
  *n_sites = (int32_t)ns;
  for (size_t k = 0; k < ns && (int32_t)k < cap; ++k) {
    if (mean_ms) mean_ms[k] = acc[k] / (double)n_steps;
    if (site_kind) site_kind[k] = sites[k].kind;
  }
  return B2B_OK;
  GUARD_END
}

b2b_status b2b_profile_graph(b2b_net* net, int64_t n_steps, double* mean_ms,
                             int32_t* site_kind, int32_t cap, int32_t* n_sites,
                             double* step_ms) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  const int K = net->cfg.steps_per_graph;
  CHECK(n_steps > 0 && n_steps % K == 0 && n_sites, B2B_ERR_INVALID_ARG,
        "n_steps must be a positive multiple of steps_per_graph (%d)", K);
  GUARD_BEGIN
  const std::vector<ProfSite> sites = profile_sites(net);
  const size_t ns = sites.size();
  // the one-CTA path advances all K steps in one launch: one timed launch per chunk
  const int marked_steps = net->small ? 1 : K;
  std::vector<cudaEvent_t> ev(2 * ns * (size_t)K, nullptr);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t nodes = 0;
  b2b_status result = B2B_OK;
  std::vector<double> acc(ns, 0.0);
  double total_ms = 0.0;
  auto cleanup = [&]() {
    net->prof_ev = nullptr;
    net->prof_sites = 0;
    if (exec) cudaGraphExecDestroy(exec);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  };
  cudaError_t e = cudaSuccess;
  for (auto& x : ev)
    if (e == cudaSuccess) e = cudaEventCreate(&x);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  if (e != cudaSuccess) {
    cleanup();
    return fail(net, B2B_ERR_CUDA, "profile events: %s", cudaGetErrorString(e));
  }
  net->prof_ev = ev.data();
  net->prof_sites = (int)ns;
  const bool use_graph = !(net->cfg.flags & B2B_NET_NO_GRAPH);
  if (use_graph) {
    const int64_t before = net->launches;
    e = cudaStreamBeginCapture(net->stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      result = enqueue_steps(net, K);
      cudaGraph_t g = nullptr;
      const cudaError_t ee = cudaStreamEndCapture(net->stream, &g);
      net->launches = before;
      if (result == B2B_OK && ee != cudaSuccess) e = ee;
      if (result == B2B_OK && e == cudaSuccess) {
        size_t nn = 0;
        cudaGraphGetNodes(g, nullptr, &nn);
        nodes = (int64_t)nn;
        e = cudaGraphInstantiate(&exec, g, 0);
      }
      if (g) cudaGraphDestroy(g);
    }
  }
  for (int64_t r = 0; result == B2B_OK && e == cudaSuccess && r < n_steps / K; ++r) {
    if ((result = refill_rng(net, K)) != B2B_OK) break;
    e = cudaEventRecord(e0, net->stream);
    if (e != cudaSuccess) break;
    if (use_graph) {
      e = cudaGraphLaunch(exec, net->stream);
      net->launches += nodes;
    } else {
      result = enqueue_steps(net, K);
    }
    if (result != B2B_OK || e != cudaSuccess) break;
    e = cudaEventRecord(e1, net->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) break;
    float ms = 0.f;
    e = cudaEventElapsedTime(&ms, e0, e1);
    total_ms += ms;
    for (int k = 0; e == cudaSuccess && k < marked_steps; ++k)
      for (size_t si = 0; e == cudaSuccess && si < ns; ++si) {
        const size_t q = ((size_t)k * ns + si) * 2;
        e = cudaEventElapsedTime(&ms, ev[q], ev[q + 1]);
        acc[si] += ms;
      }
    net->ts += K;
    net->last_chunk_steps = K;
  }
  cleanup();
  if (result != B2B_OK) return result;
  if (e != cudaSuccess) return fail(net, B2B_ERR_CUDA, "profile_graph: %s", cudaGetErrorString(e));
  *n_sites = (int32_t)ns;
  for (size_t k = 0; k < ns && (int32_t)k < cap; ++k) {
    if (mean_ms) mean_ms[k] = acc[k] / (double)n_steps;
    if (site_kind) site_kind[k] = sites[k].kind;
  }
  if (step_ms) *step_ms = total_ms / (double)n_steps;
  return B2B_OK;
  GUARD_END
}

// ---- autotuner ------------------------------------------------------------------------------
namespace {

// Puts the STDP records of a projection in post-grouped order (on_post walks contiguous
// records, on_pre reaches them through rec_of) or back in synapse order.  The live records
// and every stored copy of them (snapshots) are permuted together, so a later restore
// finds them in the order in use.
b2b_status set_record_order(b2b_net* net, Proj& pr, bool post_grouped) {
  if ((pr.dev.rec_of != nullptr) == post_grouped) return B2B_OK;
  cudaStream_t s = net->stream;
  if (post_grouped && !pr.rec_buf) {
    CU(dalloc(pr, &pr.rec_buf, (size_t)pr.n_syn));
    CU(build_rec_of(pr.dev.post_syn, pr.n_syn, pr.rec_buf, s));
  }
  const size_t bytes = 4 * real_size(pr.dtype) * (size_t)pr.n_syn;
  std::vector<void*> copies = {pr.dev.syn4};
  const auto state = state_arrays(net);
  for (size_t k = 0; k < state.size(); ++k) {
    if (state[k].first != pr.dev.syn4) continue;
    for (const Snapshot& sn : net->snapshots)
      if (sn.valid && k < sn.buffers.size()) copies.push_back(sn.buffers[k]);
  }
  void* tmp = nullptr;
  CU(cudaMalloc(&tmp, bytes ? bytes : 1));
  cudaError_t e = cudaSuccess;
  for (void* a : copies) {
    if (e == cudaSuccess)
      e = permute_stdp_records(a, tmp, pr.dev.post_syn, pr.n_syn, pr.dtype, post_grouped, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(a, tmp, bytes, cudaMemcpyDeviceToDevice, s);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(tmp);
  if (e != cudaSuccess) return fail(net, B2B_ERR_CUDA, "record order: %s", cudaGetErrorString(e));
  pr.dev.rec_of = post_grouped ? pr.rec_buf : nullptr;
  if (net->graph) {   // the graph holds the projection's parameters
    cudaGraphExecDestroy(net->graph);
    net->graph = nullptr;
  }
  return B2B_OK;
}

constexpr double kTuneMargin = 0.98;

// Launch shape of the delivery launch of a net run with two launches per step (pending.cu):
// lanes per work item (0: 8) and CTAs (0: two per SM).
// The pull form's connectivity split by the slices of sdev (cluster and slice set): for each
// rank, offsets by presynaptic neuron and slice-local targets, uploaded to the device; false
// when a slice's targets do not fit a CTA's shared memory.
bool build_pull_slices(b2b_net* net) {
  SmallDev& D = net->sdev;
  const int64_t n = net->pops[0].n, S = D.slice;
  const int C = D.cluster;
  const int P = (int)net->projs.size();
  std::vector<int32_t> hoff((size_t)P * C * (n + 1));
  std::vector<int64_t> base((size_t)P * (C + 1), 0);
  std::vector<int64_t> per_rank(C, 0);
  for (int p = 0; p < P; ++p) {
    const std::vector<int64_t>& off = net->pull_host_off[p];
    const std::vector<int32_t>& post = net->pull_host_post[p];
    std::vector<int64_t> cnt((size_t)C * (n + 1), 0);
    for (int64_t pre = 0; pre < n; ++pre)
      for (int64_t s = off[pre]; s < off[pre + 1]; ++s)
        ++cnt[(size_t)(post[s] / S) * (n + 1) + pre];
    for (int r = 0; r < C; ++r) {
      int64_t acc = 0;
      int32_t* o = hoff.data() + ((size_t)p * C + r) * (n + 1);
      for (int64_t pre = 0; pre < n; ++pre) {
        o[pre] = (int32_t)acc;
        acc += cnt[(size_t)r * (n + 1) + pre];
      }
      o[n] = (int32_t)acc;
      base[(size_t)p * (C + 1) + r + 1] = base[(size_t)p * (C + 1) + r] + acc;
      per_rank[r] += acc;
    }
  }
  // targets: projection-major, then rank, then presynaptic neuron
  std::vector<int64_t> pstart(P + 1, 0);
  for (int p = 0; p < P; ++p) pstart[p + 1] = pstart[p] + base[(size_t)p * (C + 1) + C];
  std::vector<uint16_t> htgt((size_t)std::max<int64_t>(pstart[P], 1));
  for (int p = 0; p < P; ++p) {
    const std::vector<int64_t>& off = net->pull_host_off[p];
    const std::vector<int32_t>& post = net->pull_host_post[p];
    std::vector<int32_t> fill((size_t)C * (n + 1), 0);
    for (int64_t pre = 0; pre < n; ++pre)
      for (int64_t s = off[pre]; s < off[pre + 1]; ++s) {
        const int r = (int)(post[s] / S);
        const size_t at = (size_t)(pstart[p] + base[(size_t)p * (C + 1) + r] +
                                   hoff[((size_t)p * C + r) * (n + 1) + pre] +
                                   fill[(size_t)r * (n + 1) + pre]++);
        htgt[at] = (uint16_t)(post[s] - (int64_t)r * S);
      }
    for (int r = 0; r <= C; ++r) base[(size_t)p * (C + 1) + r] += pstart[p];   // absolute
  }
  D.pull_max_tgt = (int32_t)*std::max_element(per_rank.begin(), per_rank.end());
  const size_t need = small_cluster_smem(D, net->pops[0].kind, net->pops[0].dtype);
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, net->cfg.device);
  if (optin > 0 && need > (size_t)optin - 4096) return false;
  const size_t bb = sizeof(int64_t) * base.size(), ob = sizeof(int32_t) * hoff.size();
  const size_t tb = sizeof(uint16_t) * htgt.size();
  void* buf = nullptr;
  if (cudaMalloc(&buf, bb + ob + tb) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  uint8_t* b8 = static_cast<uint8_t*>(buf);
  if (cudaMemcpy(b8, base.data(), bb, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(b8 + bb, hoff.data(), ob, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(b8 + bb + ob, htgt.data(), tb, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(buf);
    return false;
  }
  if (net->pull_buf) cudaFree(net->pull_buf);
  net->pull_buf = buf;
  D.pull_base = reinterpret_cast<const int64_t*>(b8);
  D.pull_off = reinterpret_cast<const int32_t*>(b8 + bb);
  D.pull_tgt = reinterpret_cast<const uint16_t*>(b8 + bb + ob);
  return true;
}

// The small-network path as one CTA (c == 1) or one cluster of c CTAs, each holding a slice
// of the population, pushing the effects or (pull) gathering them at the targets; false
// (nothing changed) when that form cannot run the net.
bool set_small_cluster(b2b_net* net, int c, bool pull) {
  SmallDev& D = net->sdev;
  const Pop& pop = net->pops[0];
  const int32_t c0 = D.cluster, p0 = D.pull;
  const int64_t s0 = D.slice;
  if (c == 1 && !pull) {
    D.cluster = 1;
    D.pull = 0;
    D.slice = pop.n;
  } else {
    if ((c != 8 && c != 16) || (pull && !net->pull_ok)) return false;
    D.cluster = c;
    D.pull = pull ? 1 : 0;
    D.slice = ((pop.n + c - 1) / c + 3) / 4 * 4;
    if (pull && !build_pull_slices(net)) {
      D.cluster = c0;
      D.pull = p0;
      D.slice = s0;
      return false;
    }
    if (!small_cluster_possible(D, pop.kind, pop.dtype)) {
      D.cluster = c0;
      D.pull = p0;
      D.slice = s0;
      return false;
    }
  }
  if (net->graph) {
    cudaGraphExecDestroy(net->graph);
    net->graph = nullptr;
  }
  return true;
}

void set_one_launch_grid(b2b_net* net, int grid) {
  int sms = kNumSMs;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, net->cfg.device);
  net->one_launch_grid = grid > 0 ? grid : 3 * sms / 2;   // 0: the built-in 1.5 per SM
  if (net->graph) {
    cudaGraphExecDestroy(net->graph);
    net->graph = nullptr;
  }
}

void set_pending_shape(b2b_net* net, int group, int grid) {
  int sms = kNumSMs;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, net->cfg.device);
  net->pending_grid = grid > 0 ? grid : 2 * sms;
  net->pdev.group = group > 0 ? group : 8;
  if (net->graph) {
    cudaGraphExecDestroy(net->graph);
    net->graph = nullptr;
  }
}

// Advances the net by n_steps the way b2b_run does (CUDA-graph replays of the current launch
// shapes, captured afresh before the timing starts), timed with a CUDA event pair on the
// net's stream; *mean_ms receives the mean device time of one whole step.  A shape is judged
// by the step it produces, so its effect on the neighbouring launches (a larger grid delays
// the next kernel's start) counts too.
b2b_status time_steps(b2b_net* net, int64_t n_steps, double* mean_ms) {
  if (net->graph) {
    cudaGraphExecDestroy(net->graph);
    net->graph = nullptr;
  }
  if (!(net->cfg.flags & B2B_NET_NO_GRAPH))
    if (b2b_status st = capture_graph(net)) return st;
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  cudaEventRecord(e0, net->stream);
  b2b_status st = b2b_run(net, n_steps);
  cudaEventRecord(e1, net->stream);
  cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.f;
  if (st == B2B_OK && e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != B2B_OK) return st;
  if (e != cudaSuccess) return fail(net, B2B_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
  *mean_ms = ms / (double)n_steps;
  return B2B_OK;
}

}  // namespace

b2b_status b2b_autotune(b2b_net* net, int32_t trial_steps, b2b_tune_result* out, int32_t cap,
                        int32_t* n_out) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  CHECK(trial_steps > 0 && trial_steps <= 100000 && n_out, B2B_ERR_INVALID_ARG, "bad arguments");
  GUARD_BEGIN
  CU(cudaStreamSynchronize(net->stream));
  // the state to start every trial from, in a slot of its own; monitor counts to put back
  const int slot = (int)net->snapshots.size();
  if (b2b_status st = b2b_store(net, slot)) return st;
  std::vector<unsigned long long> mon(net->pops.size(), 0);
  for (size_t p = 0; p < net->pops.size(); ++p)
    if (net->pops[p].dev.mon_cnt)
      CU(cudaMemcpy(&mon[p], net->pops[p].dev.mon_cnt, sizeof(unsigned long long),
                    cudaMemcpyDeviceToHost));
  std::vector<unsigned long long> smon(net->smons.size()), rmon(net->rmons.size());
  for (size_t m = 0; m < net->smons.size(); ++m)
    CU(cudaMemcpy(&smon[m], net->smons[m].dev.cnt, sizeof(unsigned long long),
                  cudaMemcpyDeviceToHost));
  for (size_t m = 0; m < net->rmons.size(); ++m)
    CU(cudaMemcpy(&rmon[m], net->rmons[m].dev.cnt, sizeof(unsigned long long),
                  cudaMemcpyDeviceToHost));
  net->add_tune.resize(net->add_batches.size());
  std::vector<b2b_tune_result> res;
  b2b_status st = B2B_OK;
  auto put_back_monitors = [&]() -> b2b_status {
    for (size_t p = 0; p < net->pops.size(); ++p)
      if (net->pops[p].dev.mon_cnt)
        CU(cudaMemcpy(net->pops[p].dev.mon_cnt, &mon[p], sizeof(unsigned long long),
                      cudaMemcpyHostToDevice));
    for (size_t m = 0; m < net->smons.size(); ++m)
      CU(cudaMemcpy(net->smons[m].dev.cnt, &smon[m], sizeof(unsigned long long),
                    cudaMemcpyHostToDevice));
    for (size_t m = 0; m < net->rmons.size(); ++m)
      CU(cudaMemcpy(net->rmons[m].dev.cnt, &rmon[m], sizeof(unsigned long long),
                    cudaMemcpyHostToDevice));
    return B2B_OK;
  };
  // every trial starts from the same state, with the monitors' counts of that state
  auto trial = [&](double* ms) {
    if (b2b_status s2 = b2b_restore(net, slot)) return s2;
    if (b2b_status s2 = put_back_monitors()) return s2;
    return time_steps(net, trial_steps, ms);
  };
  // one discarded trial first, so that no candidate pays for a cold start (first launches,
  // caches, clocks ramping up)
  {
    double ms = 0;
    st = trial(&ms);
  }
  if (net->small) {
    // the small-network path: one CTA, or one thread-block cluster of 8 or 16 CTAs pushing
    // the effects or pulling them at the targets
    SmallDev& D = net->sdev;
    const int32_t c0 = D.cluster, p0 = D.pull;
    b2b_tune_result r{14, 0, c0, p0, 0.0, 0.0};
    double best = 1e30;
    const std::pair<int, int> forms[] = {{c0, p0}, {1, 0}, {8, 0}, {16, 0}, {8, 1}, {16, 1}};
    for (int c = 0; c < 6 && st == B2B_OK; ++c) {
      if (c > 0 && forms[c].first == c0 && forms[c].second == p0) continue;
      if (!set_small_cluster(net, forms[c].first, forms[c].second != 0)) continue;
      double ms = 0;
      st = trial(&ms);
      if (c == 0) r.default_ms = ms;
      if (st == B2B_OK && (c == 0 || ms < kTuneMargin * best)) {
        best = ms;
        r.choice_a = forms[c].first;
        r.choice_b = forms[c].second;
      }
    }
    set_small_cluster(net, r.choice_a, r.choice_b != 0);
    r.best_ms = best;
    res.push_back(r);
  } else {
    int sms = kNumSMs;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, net->cfg.device);
    // a net that allows both forms of the step tunes the per-step kernels first, then the two
    // concurrent launches, and keeps the faster form
    const bool builtin_two_launch = net->two_launch;
    const bool builtin_one_launch = net->two_launch && net->one_launch;
    if (net->two_launch_ok) net->two_launch = false;
    net->one_launch = false;
    for (size_t p = 0; p < net->pops.size() && st == B2B_OK && !net->two_launch; ++p) {
      Pop& pop = net->pops[p];
      if (pop.kind == KIND_SPIKEGEN || pop.kind == KIND_MODEL) continue;
      std::vector<std::pair<int, int>> cands;   // (a, b); the first is the built-in choice
      if (pop.surr_img) {
        cands = {{0, 0}, {2, 0}, {3, 0}, {4, 0}, {6, 0}};
      } else {
        cands = {{0, 0}, {1, 128}, {1, 256}, {2, 128}, {2, 256}, {4, 128}, {4, 256}};
      }
      b2b_tune_result r{1, (int32_t)p, 0, 0, 0.0, 0.0};
      double best = 1e30;
      for (size_t c = 0; c < cands.size() && st == B2B_OK; ++c) {
        if (pop.surr_img) {
          pop.tune_ctas = cands[c].first;
        } else {
          pop.tune_e = cands[c].first;
          pop.tune_block = cands[c].second;
        }
        double ms = 0;
        st = trial(&ms);
        if (c == 0) r.default_ms = ms;
        // a candidate replaces the built-in shape only when it is 2 % faster: trial times of
        // near-equal shapes differ by noise, and noise should not pick the shape
        if (st == B2B_OK && (c == 0 ? true : ms < kTuneMargin * best)) {
          best = ms;
          r.choice_a = cands[c].first;
          r.choice_b = cands[c].second;
        }
      }
      if (pop.surr_img) {
        pop.tune_ctas = r.choice_a;
      } else {
        pop.tune_e = r.choice_a;
        pop.tune_block = r.choice_b;
      }
      r.best_ms = best;
      res.push_back(r);
    }
    for (size_t b = 0; b < net->add_batches.size() && st == B2B_OK && !net->two_launch; ++b) {
      AddTune& t = net->add_tune[b];
      std::vector<std::pair<int, int>> cands = {{0, 0}};
      for (int g : {2, 4, 8, 16, 32})
        for (int mult : {1, 2, 4, 8, 16}) cands.push_back({g, mult * sms / 2});
      b2b_tune_result r{6, (int32_t)b, 0, 0, 0.0, 0.0};
      double best = 1e30;
      for (size_t c = 0; c < cands.size() && st == B2B_OK; ++c) {
        t.group = cands[c].first;
        t.grid = cands[c].second;
        double ms = 0;
        st = trial(&ms);
        if (c == 0) r.default_ms = ms;
        // a candidate replaces the built-in shape only when it is 2 % faster: trial times of
        // near-equal shapes differ by noise, and noise should not pick the shape
        if (st == B2B_OK && (c == 0 ? true : ms < kTuneMargin * best)) {
          best = ms;
          r.choice_a = cands[c].first;
          r.choice_b = cands[c].second;
        }
      }
      t.group = r.choice_a;
      t.grid = r.choice_b;
      r.best_ms = best;
      res.push_back(r);
    }
    // additive delivery launches that can accumulate in thread-block clusters (float32, one
    // target population): with the chosen lanes per item, cluster accumulation on or off
    for (size_t b = 0; b < net->add_batches.size() && st == B2B_OK && !net->two_launch; ++b) {
      const auto& bat = net->add_batches[b];
      if (!add_batch_cluster_capable(bat.data(), (int)bat.size())) continue;
      AddTune& t = net->add_tune[b];
      b2b_tune_result r{12, (int32_t)b, 0, 0, 0.0, 0.0};
      double off_ms = 0, on_ms = 0;
      t.cluster = 0;
      st = trial(&off_ms);
      if (st != B2B_OK) break;
      t.cluster = 1;
      st = trial(&on_ms);
      const bool use = st == B2B_OK && on_ms < kTuneMargin * off_ms;
      t.cluster = use ? 1 : 0;
      r.choice_a = t.cluster;
      r.default_ms = off_ms;
      r.best_ms = use ? on_ms : off_ms;
      res.push_back(r);
    }
    if (net->two_launch_ok && st == B2B_OK) {
      const double per_step_ms = res.empty() ? 1e30 : res.back().best_ms;
      net->two_launch = true;
      // the step's delivery launch: lanes per work item x CTAs (the neuron launch has one
      // thread per neuron)
      std::vector<std::pair<int, int>> cands = {{0, 0}};
      for (int g : {2, 4, 8, 16})
        for (int mult : {1, 2, 4}) cands.push_back({g, mult * sms / 2});
      b2b_tune_result r{5, 0, 0, 0, 0.0, 0.0};
      double best = 1e30;
      for (size_t c = 0; c < cands.size() && st == B2B_OK; ++c) {
        set_pending_shape(net, cands[c].first, cands[c].second);
        double ms = 0;
        st = trial(&ms);
        if (c == 0) r.default_ms = ms;
        if (st == B2B_OK && (c == 0 ? true : ms < kTuneMargin * best)) {
          best = ms;
          r.choice_a = cands[c].first;
          r.choice_b = cands[c].second;
        }
      }
      set_pending_shape(net, r.choice_a, r.choice_b);
      r.best_ms = best;
      res.push_back(r);
      // the update's shape again, inside this form: the per-step form tuned it for an update
      // followed by its own delivery, and the forms rank the shapes differently (COBAHH 1e5:
      // 1 x 256 against 2 x 128 neurons per thread x threads, 45.8 against 37.7 ms per
      // simulated second with two launches)
      Pop& pop0 = net->pops[0];
      const int ps_e = pop0.tune_e, ps_block = pop0.tune_block;
      b2b_tune_result r1{1, 0, ps_e, ps_block, best, best};
      {
        const std::pair<int, int> shapes[] = {{0, 0}, {1, 128}, {1, 256}, {2, 128}, {2, 256},
                                              {4, 128}, {4, 256}};
        for (const auto& sh : shapes) {
          if (st != B2B_OK) break;
          if (sh.first == ps_e && sh.second == ps_block) continue;   // timed above
          pop0.tune_e = sh.first;
          pop0.tune_block = sh.second;
          set_pending_shape(net, r.choice_a, r.choice_b);   // a fresh graph
          double ms = 0;
          st = trial(&ms);
          if (st == B2B_OK && ms < kTuneMargin * r1.best_ms) {
            r1.best_ms = ms;
            r1.choice_a = sh.first;
            r1.choice_b = sh.second;
          }
        }
        pop0.tune_e = r1.choice_a;
        pop0.tune_block = r1.choice_b;
        set_pending_shape(net, r.choice_a, r.choice_b);
      }
      const double two_launch_ms = r1.best_ms;
      // the same halves as one grid per step: CTAs of the delivery after the update's
      double one_launch_ms = 1e30;
      int one_grid = 3 * sms / 2;
      const int two_group = net->pdev.group;
      int one_group = two_group;
      if (net->one_launch_ok && st == B2B_OK) {
        net->one_launch = true;
        // the built-in 1.5 per SM first: between 1 and 2 per SM the delivering CTAs still fit
        // beside the update's in one wave (COBAHH 1e5, update 2 x 128: 148, 185, 222, 259 gave
        // 38.1, 37.4, 36.9, 37.8 ms per simulated second on one box, 148 against 222 38.1
        // against 37.2 on another; 296 needs a second wave), and the 2000-step window does not
        // tell 1 and 1.5 per SM apart by the 2 % margin
        const int grids[] = {3 * sms / 2, net->pending_grid, sms / 2, sms, 5 * sms / 4,
                             7 * sms / 4, 2 * sms, 4 * sms};
        auto tune_grid = [&](bool first) {
          for (size_t c = 0; c < sizeof(grids) / sizeof(grids[0]) && st == B2B_OK; ++c) {
            if (!first && grids[c] == one_grid) continue;   // timed already
            set_one_launch_grid(net, grids[c]);
            double ms = 0;
            st = trial(&ms);
            if (st == B2B_OK && ((first && c == 0) || ms < kTuneMargin * one_launch_ms)) {
              one_launch_ms = ms;
              one_grid = grids[c];
            }
          }
          set_one_launch_grid(net, one_grid);
        };
        tune_grid(true);
        // lanes per work item inside this form: its delivering CTAs share the SMs with the
        // update's, and a population burst's delivery is many short bundles, so the form
        // ranks them differently from the two launches (COBAHH 1e5: 4 lanes 37.0-37.4
        // against 16 lanes 39.7 ms per simulated second, on one box)
        const int groups[] = {2, 4, 8, 16};
        for (int g : groups) {
          if (g == two_group || st != B2B_OK) continue;
          net->pdev.group = g;
          set_one_launch_grid(net, one_grid);
          double ms = 0;
          st = trial(&ms);
          if (st == B2B_OK && ms < kTuneMargin * one_launch_ms) {
            one_launch_ms = ms;
            one_group = g;
          }
        }
        net->pdev.group = one_group;
        if (one_group != two_group) tune_grid(false);   // the CTAs again, for these lanes
        // the update's CTAs inside this form (one or two neurons per thread x 128 or 256
        // threads): they share the grid with the delivery's, and fewer, larger CTAs shorten
        // the launch
        const std::pair<int, int> one_shapes[] = {{1, 128}, {1, 256}, {2, 128}, {2, 256}};
        auto eff = [](int e, int b) {
          return std::make_pair(e == 2 || e == 4 ? 2 : 1, b > 0 ? b : kBlock);
        };
        const auto cur = eff(pop0.tune_e, pop0.tune_block);
        for (const auto& sh : one_shapes) {
          if (sh == cur || st != B2B_OK) continue;
          const int pe = pop0.tune_e, pb = pop0.tune_block;
          pop0.tune_e = sh.first;
          pop0.tune_block = sh.second;
          set_one_launch_grid(net, one_grid);
          double ms = 0;
          st = trial(&ms);
          if (st == B2B_OK && ms < kTuneMargin * one_launch_ms) {
            one_launch_ms = ms;
          } else {
            pop0.tune_e = pe;
            pop0.tune_block = pb;
          }
        }
        set_one_launch_grid(net, one_grid);
      }
      const int one_e = pop0.tune_e, one_block = pop0.tune_block;
      // the same, each step's launch chained to the previous one (programmatic dependent launch)
      double chained_ms = 1e30;
      if (net->one_launch_ok && st == B2B_OK) {
        net->one_launch_chained = true;
        set_one_launch_grid(net, one_grid);
        st = trial(&chained_ms);
        net->one_launch_chained = false;
        set_one_launch_grid(net, one_grid);
      }
      net->one_launch = false;
      // the form of the step: 0 per-step kernels, 1 two concurrent launches, 2 one launch, 3 one
      // launch chained; the built-in form stays unless another is 2 % faster
      const double form_ms[4] = {per_step_ms, two_launch_ms, one_launch_ms, chained_ms};
      const int builtin = builtin_two_launch ? (builtin_one_launch ? 2 : 1) : 0;
      int other = -1;
      for (int f = 0; f < 4; ++f)
        if (f != builtin && (other < 0 || form_ms[f] < form_ms[other])) other = f;
      const int form = form_ms[other] < kTuneMargin * form_ms[builtin] ? other : builtin;
      net->two_launch = form >= 1;
      net->one_launch = form >= 2;
      net->one_launch_chained = form == 3;
      if (form == 0) {
        // the per-step form keeps the shape tuned for it
        pop0.tune_e = ps_e;
        pop0.tune_block = ps_block;
      } else {
        if (r1.choice_a != ps_e || r1.choice_b != ps_block)
          res.push_back(r1);   // after the per-step form's entry, so that tune_apply ends on it
        pop0.tune_e = r1.choice_a;
        pop0.tune_block = r1.choice_b;
        if (form >= 2 && (one_e != r1.choice_a || one_block != r1.choice_b)) {
          pop0.tune_e = one_e;
          pop0.tune_block = one_block;
          res.push_back(b2b_tune_result{1, 0, one_e, one_block, form_ms[form], r1.best_ms});
        }
      }
      set_pending_shape(net, r.choice_a, r.choice_b);
      if (form >= 2 && one_group != two_group) {
        // the one-launch form's lanes per item (the pending delivery's CTAs stay as tuned)
        set_pending_shape(net, one_group, r.choice_b);
        res.push_back(b2b_tune_result{5, 0, one_group, r.choice_b, form_ms[form], r.best_ms});
      }
      res.push_back(b2b_tune_result{11, 0, form, form >= 2 ? one_grid : 0, form_ms[form],
                                    form_ms[builtin]});
    }
    // STDP projections: order of the synapse records (0 synapse order, 1 post-grouped)
    for (size_t p = 0; p < net->projs.size() && st == B2B_OK; ++p) {
      Proj& pr = net->projs[p];
      if (pr.effect != B2B_EFFECT_STDP) continue;
      b2b_tune_result r{8, (int32_t)p, 0, 0, 0.0, 0.0};
      double best = 1e30;
      for (int c = 0; c < 2 && st == B2B_OK; ++c) {
        st = set_record_order(net, pr, c == 1);
        double ms = 0;
        if (st == B2B_OK) st = trial(&ms);
        if (c == 0) r.default_ms = ms;
        if (st == B2B_OK && (c == 0 || ms < kTuneMargin * best)) {
          best = ms;
          r.choice_a = c;
        }
      }
      if (st == B2B_OK) st = set_record_order(net, pr, r.choice_a == 1);
      r.best_ms = best;
      res.push_back(r);
    }
    if (st != B2B_OK && net->two_launch_ok) {
      net->two_launch = builtin_two_launch;
      net->one_launch = builtin_one_launch;
      net->one_launch_chained = false;
    }
    // a net that allows the small-network path: its forms against the step as tuned above
    if (net->small_ok && st == B2B_OK) {
      double base_ms = 0;
      st = trial(&base_ms);
      b2b_tune_result r{14, 0, 0, 0, base_ms, base_ms};
      const std::pair<int, int> forms[] = {{1, 0}, {8, 0}, {16, 0}, {8, 1}, {16, 1}};
      for (const auto& f : forms) {
        if (st != B2B_OK) break;
        net->small = true;
        if (!set_small_cluster(net, f.first, f.second != 0)) continue;
        double ms = 0;
        st = trial(&ms);
        if (st == B2B_OK && ms < kTuneMargin * r.best_ms) {
          r.best_ms = ms;
          r.choice_a = f.first;
          r.choice_b = f.second;
        }
      }
      net->small = r.choice_a > 0;
      if (net->small) set_small_cluster(net, r.choice_a, r.choice_b != 0);
      if (net->graph) {
        cudaGraphExecDestroy(net->graph);
        net->graph = nullptr;
      }
      res.push_back(r);
    }
  }
  // back to the starting state; the next b2b_run captures a graph with the chosen shapes
  b2b_status st2 = b2b_restore(net, slot);
  if (st2 == B2B_OK) st2 = put_back_monitors();
  for (void* a : net->snapshots[slot].buffers) cudaFree(a);
  net->snapshots.resize(slot);
  if (net->graph) {
    cudaGraphExecDestroy(net->graph);
    net->graph = nullptr;
  }
  if (st != B2B_OK) return st;
  if (st2 != B2B_OK) return st2;
  *n_out = (int32_t)res.size();
  for (size_t k = 0; k < res.size() && (int32_t)k < cap; ++k)
    if (out) out[k] = res[k];
  return B2B_OK;
  GUARD_END
}

b2b_status b2b_tune_apply(b2b_net* net, const b2b_tune_result* r, int32_t n) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  CHECK(n >= 0 && (r || n == 0), B2B_ERR_INVALID_ARG, "bad arguments");
  net->add_tune.resize(net->add_batches.size());
  for (int32_t k = 0; k < n; ++k) {
    const b2b_tune_result& t = r[k];
    if (t.site_kind == 1) {
      CHECK(t.site_index >= 0 && t.site_index < (int32_t)net->pops.size(), B2B_ERR_INVALID_ARG,
            "bad population index %d", t.site_index);
      Pop& pop = net->pops[t.site_index];
      if (pop.surr_img) {
        CHECK(t.choice_a >= 0 && t.choice_a <= 8, B2B_ERR_INVALID_ARG, "bad CTAs per SM");
        pop.tune_ctas = t.choice_a;
      } else {
        CHECK((t.choice_a == 0 || t.choice_a == 1 || t.choice_a == 2 || t.choice_a == 4) &&
                  (t.choice_b == 0 || t.choice_b == 128 || t.choice_b == 256),
              B2B_ERR_INVALID_ARG, "bad neuron launch shape");
        pop.tune_e = t.choice_a;
        pop.tune_block = t.choice_b;
      }
    } else if (t.site_kind == 6) {
      CHECK(t.site_index >= 0 && t.site_index < (int32_t)net->add_batches.size(),
            B2B_ERR_INVALID_ARG, "bad delivery launch index %d", t.site_index);
      CHECK((t.choice_a == 0 || t.choice_a == 2 || t.choice_a == 4 || t.choice_a == 8 ||
             t.choice_a == 16 || t.choice_a == 32) &&
                t.choice_b >= 0 && t.choice_b <= 65535,
            B2B_ERR_INVALID_ARG, "bad delivery launch shape");
      net->add_tune[t.site_index].group = t.choice_a;
      net->add_tune[t.site_index].grid = t.choice_b;
    } else if (t.site_kind == 12) {
      CHECK(t.site_index >= 0 && t.site_index < (int32_t)net->add_batches.size() &&
                (t.choice_a == 0 || t.choice_a == 1),
            B2B_ERR_INVALID_ARG, "bad cluster choice for delivery launch %d", t.site_index);
      const auto& bat = net->add_batches[t.site_index];
      CHECK(t.choice_a == 0 || add_batch_cluster_capable(bat.data(), (int)bat.size()),
            B2B_ERR_UNSUPPORTED, "delivery launch %d cannot accumulate in clusters",
            t.site_index);
      net->add_tune[t.site_index].cluster = t.choice_a;
    } else if (t.site_kind == 11) {
      CHECK(net->two_launch_ok && t.site_index == 0 && t.choice_a >= 0 && t.choice_a <= 3,
            B2B_ERR_INVALID_ARG, "site kind 11 exists only for nets that allow both step forms");
      CHECK(t.choice_a < 2 || (net->one_launch_ok && t.choice_b >= 0 && t.choice_b <= 65535),
            B2B_ERR_INVALID_ARG, "the net does not allow the one-launch step");
      net->two_launch = t.choice_a >= 1;
      net->one_launch = t.choice_a >= 2;
      net->one_launch_chained = t.choice_a == 3;
      if (t.choice_a >= 2) set_one_launch_grid(net, t.choice_b);
    } else if (t.site_kind == 5) {
      CHECK(net->two_launch_ok && t.site_index == 0, B2B_ERR_INVALID_ARG,
            "site kind 5 exists only for nets that allow two launches per step");
      CHECK((t.choice_a == 0 || t.choice_a == 2 || t.choice_a == 4 || t.choice_a == 8 ||
             t.choice_a == 16) &&
                t.choice_b >= 0 && t.choice_b <= 65535,
            B2B_ERR_INVALID_ARG, "bad delivery launch shape");
      set_pending_shape(net, t.choice_a, t.choice_b);
    } else if (t.site_kind == 14) {
      CHECK(net->small_ok && t.site_index == 0, B2B_ERR_INVALID_ARG,
            "site kind 14 exists only for a net that allows the small-network path");
      CHECK(t.choice_b == 0 || t.choice_b == 1, B2B_ERR_INVALID_ARG, "bad small-path form");
      CHECK(t.choice_a != 0 || !(net->cfg.flags & B2B_NET_SMALL), B2B_ERR_INVALID_ARG,
            "B2B_NET_SMALL keeps the small-network path");
      if (t.choice_a == 0) {
        net->small = false;
        if (net->graph) {
          cudaGraphExecDestroy(net->graph);
          net->graph = nullptr;
        }
      } else {
        const bool was = net->small;
        net->small = true;
        if (!set_small_cluster(net, t.choice_a, t.choice_b == 1)) {
          net->small = was;
          CHECK(false, B2B_ERR_UNSUPPORTED, "the small-network path cannot run as %d CTAs%s here",
                t.choice_a, t.choice_b == 1 ? " pulling the effects" : "");
        }
      }
    } else if (t.site_kind == 8) {
      CHECK(t.site_index >= 0 && t.site_index < (int32_t)net->projs.size() &&
                net->projs[t.site_index].effect == B2B_EFFECT_STDP,
            B2B_ERR_INVALID_ARG, "bad STDP projection index %d", t.site_index);
      CHECK(t.choice_a == 0 || t.choice_a == 1, B2B_ERR_INVALID_ARG, "bad record order");
      if (b2b_status st = set_record_order(net, net->projs[t.site_index], t.choice_a == 1))
        return st;
    } else {
      return fail(net, B2B_ERR_INVALID_ARG, "bad site kind %d", t.site_kind);
    }
  }
  if (net->graph) {
    cudaGraphExecDestroy(net->graph);
    net->graph = nullptr;
  }
  return B2B_OK;
}

b2b_status b2b_sync(b2b_net* net, int32_t* device_status) {
  if (b2b_status st = check_net(net)) return st;
  CU(cudaStreamSynchronize(net->stream));
  int32_t s = 0;
  CU(cudaMemcpy(&s, net->d_status, sizeof(int32_t), cudaMemcpyDeviceToHost));
  if (device_status) *device_status = s;
  return B2B_OK;
}

b2b_status b2b_store(b2b_net* net, int32_t slot) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  CHECK(slot >= 0 && slot < 1024, B2B_ERR_INVALID_ARG, "bad slot %d", slot);
  GUARD_BEGIN
  if ((int)net->snapshots.size() <= slot) net->snapshots.resize(slot + 1);
  Snapshot& sn = net->snapshots[slot];
  const auto arrays = state_arrays(net);
  if (sn.buffers.size() != arrays.size()) {
    for (void* p : sn.buffers) cudaFree(p);
    sn.buffers.assign(arrays.size(), nullptr);
    for (size_t k = 0; k < arrays.size(); ++k) CU(cudaMalloc(&sn.buffers[k], arrays[k].second));
  }
  for (size_t k = 0; k < arrays.size(); ++k)
    CU(cudaMemcpyAsync(sn.buffers[k], arrays[k].first, arrays[k].second,
                       cudaMemcpyDeviceToDevice, net->stream));
  CU(cudaStreamSynchronize(net->stream));
  sn.ts = net->ts;
  sn.rng_offset = net->rng_offset;
  sn.valid = true;
  return B2B_OK;
  GUARD_END
}

b2b_status b2b_restore(b2b_net* net, int32_t slot) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(slot >= 0 && slot < (int)net->snapshots.size() && net->snapshots[slot].valid,
        B2B_ERR_INVALID_ARG, "no checkpoint in slot %d", slot);
  const Snapshot& sn = net->snapshots[slot];
  const auto arrays = state_arrays(net);
  for (size_t k = 0; k < arrays.size(); ++k)
    CU(cudaMemcpyAsync(arrays[k].first, sn.buffers[k], arrays[k].second,
                       cudaMemcpyDeviceToDevice, net->stream));
  net->ts = sn.ts;
  CU(cudaMemcpyAsync(net->d_clock, &net->ts, sizeof(int64_t), cudaMemcpyHostToDevice,
                     net->stream));
  CU(cudaStreamSynchronize(net->stream));
  if (net->gen && net->rng_offset != sn.rng_offset) {
    if (curandSetGeneratorOffset(net->gen, sn.rng_offset) != CURAND_STATUS_SUCCESS)
      return fail(net, B2B_ERR_CUDA, "curandSetGeneratorOffset failed");
    net->rng_offset = sn.rng_offset;
  }
  return B2B_OK;
}

b2b_status b2b_time(b2b_net* net, int64_t* timestep, double* t) {
  if (!net) return B2B_ERR_INVALID_ARG;
  if (timestep) *timestep = net->ts;
  if (t) *t = (double)net->ts * net->cfg.dt;
  return B2B_OK;
}

b2b_status b2b_run_mode(b2b_net* net, int32_t* mode) {
  if (!net || !mode) return B2B_ERR_INVALID_ARG;
  if (!net->finalized) return fail(net, B2B_ERR_STATE, "call b2b_finalize first");
  *mode = net->small ? 2 : (net->two_launch ? (net->one_launch ? 3 : 1) : 0);
  return B2B_OK;
}

b2b_status b2b_kernel_launches(b2b_net* net, int64_t* n) {
  if (!net || !n) return B2B_ERR_INVALID_ARG;
  *n = net->launches;
  return B2B_OK;
}

b2b_status b2b_spikemon_get(b2b_net* net, int32_t gid, int64_t* n, int32_t* idx,
                            int64_t* step, int64_t cap) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(gid >= 0 && gid < (int)net->groups.size(), B2B_ERR_INVALID_ARG, "bad group %d", gid);
  return b2b_spikemon_get_range(net, gid, 0, net->groups[gid].n, n, idx, step, cap);
}

b2b_status b2b_spikemon_get_range(b2b_net* net, int32_t gid, int64_t lo, int64_t hi,
                                  int64_t* n, int32_t* idx, int64_t* step, int64_t cap) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(gid >= 0 && gid < (int)net->groups.size(), B2B_ERR_INVALID_ARG, "bad group %d", gid);
  CHECK(n != nullptr, B2B_ERR_INVALID_ARG, "n is NULL");
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  const Group& g = net->groups[gid];
  CHECK(g.mon_cap > 0, B2B_ERR_STATE, "group %d has no spike monitor", gid);
  CHECK(0 <= lo && lo <= hi && hi <= g.n, B2B_ERR_INVALID_ARG,
        "bad subgroup [%lld, %lld) of a %lld-neuron group", (long long)lo, (long long)hi,
        (long long)g.n);
  GUARD_BEGIN
  const PopDev& D = net->pops[g.pop].dev;
  CU(cudaStreamSynchronize(net->stream));
  unsigned long long total = 0;
  CU(cudaMemcpy(&total, D.mon_cnt, sizeof(total), cudaMemcpyDeviceToHost));
  const int64_t m = std::min<int64_t>((int64_t)total, D.mon_cap);
  std::vector<int32_t> midx(m);
  std::vector<int64_t> mstep(m);
  if (m) {
    CU(cudaMemcpy(midx.data(), D.mon_idx, 4 * m, cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(mstep.data(), D.mon_step, 8 * m, cudaMemcpyDeviceToHost));
  }
  std::vector<std::pair<int64_t, int32_t>> ent;
  for (int64_t k = 0; k < m; ++k)
    if (midx[k] >= g.offset + lo && midx[k] < g.offset + hi)
      ent.emplace_back(mstep[k], (int32_t)(midx[k] - g.offset - lo));
  std::sort(ent.begin(), ent.end());
  *n = (int64_t)ent.size();
  for (int64_t k = 0; k < (int64_t)ent.size() && k < cap; ++k) {
    if (idx) idx[k] = ent[k].second;
    if (step) step[k] = ent[k].first;
  }
  if ((int64_t)total > D.mon_cap)
    return fail(net, B2B_ERR_QUEUE_OVERFLOW, "spike monitor overflowed (%llu > %lld)",
                total, (long long)D.mon_cap);
  return B2B_OK;
  GUARD_END
}

namespace {
b2b_status spikemon_fetch(b2b_net* net, int32_t gid, int64_t start, int64_t* total, int64_t* n,
                          int32_t* idx, int64_t* step, int64_t cap, bool whole_population);
}  // namespace

b2b_status b2b_spikemon_fetch(b2b_net* net, int32_t gid, int64_t start, int64_t* total,
                              int64_t* n, int32_t* idx, int64_t* step, int64_t cap) {
  return spikemon_fetch(net, gid, start, total, n, idx, step, cap, false);
}

b2b_status b2b_spikemon_fetch_population(b2b_net* net, int32_t gid, int64_t start,
                                         int64_t* total, int64_t* n, int32_t* idx,
                                         int64_t* step, int64_t cap) {
  return spikemon_fetch(net, gid, start, total, n, idx, step, cap, true);
}

b2b_status b2b_group_offset(b2b_net* net, int32_t gid, int64_t* offset) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  CHECK(gid >= 0 && gid < (int)net->groups.size() && offset, B2B_ERR_INVALID_ARG, "bad arguments");
  *offset = net->groups[gid].offset;
  return B2B_OK;
}

namespace {
b2b_status spikemon_fetch(b2b_net* net, int32_t gid, int64_t start, int64_t* total, int64_t* n,
                          int32_t* idx, int64_t* step, int64_t cap, bool whole_population) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(gid >= 0 && gid < (int)net->groups.size(), B2B_ERR_INVALID_ARG, "bad group %d", gid);
  CHECK(total && n && start >= 0 && cap >= 0, B2B_ERR_INVALID_ARG, "bad arguments");
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  const Group& g = net->groups[gid];
  CHECK(g.mon_cap > 0, B2B_ERR_STATE, "group %d has no spike monitor", gid);
  const PopDev& D = net->pops[g.pop].dev;
  unsigned long long rec = 0;
  CU(cudaMemcpyAsync(&rec, D.mon_cnt, sizeof(rec), cudaMemcpyDeviceToHost, net->stream));
  CU(cudaStreamSynchronize(net->stream));
  *total = (int64_t)rec;
  *n = 0;
  const int64_t stored = std::min<int64_t>((int64_t)rec, D.mon_cap);
  const int64_t hi = std::min<int64_t>(stored, start + cap);
  if (hi <= start) return B2B_OK;
  const int64_t m = hi - start;
  // through pinned host memory kept by the net: a copy into pageable memory is staged by the
  // driver at a fraction of the link's rate (3e5 spikes: 1.6 ms against ~0.3 ms)
  const size_t need = 12 * (size_t)m;
  if (need > net->fetch_pinned_bytes) {
    if (net->fetch_pinned) cudaFreeHost(net->fetch_pinned);
    net->fetch_pinned = nullptr;
    net->fetch_pinned_bytes = 0;
    const size_t bytes = std::max(need, (size_t)1 << 20);
    CU(cudaMallocHost(&net->fetch_pinned, bytes));
    net->fetch_pinned_bytes = bytes;
  }
  int64_t* sstep = static_cast<int64_t*>(net->fetch_pinned);
  int32_t* sidx = reinterpret_cast<int32_t*>(sstep + m);
  CU(cudaMemcpyAsync(sidx, D.mon_idx + start, 4 * m, cudaMemcpyDeviceToHost, net->stream));
  CU(cudaMemcpyAsync(sstep, D.mon_step + start, 8 * m, cudaMemcpyDeviceToHost, net->stream));
  CU(cudaStreamSynchronize(net->stream));
  int64_t k = m;
  if (whole_population) {
    std::memcpy(idx, sidx, 4 * (size_t)m);
    std::memcpy(step, sstep, 8 * (size_t)m);
  } else {
    k = 0;
    for (int64_t r = 0; r < m; ++r) {
      if (sidx[r] < g.offset || sidx[r] >= g.offset + g.n) continue;
      idx[k] = (int32_t)(sidx[r] - g.offset);
      step[k] = sstep[r];
      ++k;
    }
  }
  *n = k;
  if ((int64_t)rec > D.mon_cap)
    return fail(net, B2B_ERR_QUEUE_OVERFLOW, "spike monitor overflowed");
  return B2B_OK;
}
}  // namespace

b2b_status b2b_spikes_last(b2b_net* net, int32_t gid, int64_t* n, int32_t* idx, int64_t cap) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(gid >= 0 && gid < (int)net->groups.size(), B2B_ERR_INVALID_ARG, "bad group %d", gid);
  CHECK(n != nullptr, B2B_ERR_INVALID_ARG, "n is NULL");
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  GUARD_BEGIN
  const Group& g = net->groups[gid];
  const PopDev& D = net->pops[g.pop].dev;
  *n = 0;
  if (net->ts == 0) return B2B_OK;
  CU(cudaStreamSynchronize(net->stream));
  const int slot = (int)((net->ts - 1) % D.ring_len);
  int32_t cnt = 0;
  CU(cudaMemcpy(&cnt, D.ring_cnt + slot, 4, cudaMemcpyDeviceToHost));
  std::vector<int32_t> h(cnt);
  if (cnt) CU(cudaMemcpy(h.data(), D.ring_idx + (int64_t)slot * D.n, 4 * (size_t)cnt,
                         cudaMemcpyDeviceToHost));
  std::vector<int32_t> mine;
  for (int32_t x : h)
    if (x >= g.offset && x < g.offset + g.n) mine.push_back((int32_t)(x - g.offset));
  std::sort(mine.begin(), mine.end());
  *n = (int64_t)mine.size();
  if (idx)
    for (int64_t k = 0; k < (int64_t)mine.size() && k < cap; ++k) idx[k] = mine[k];
  return B2B_OK;
  GUARD_END
}

b2b_status b2b_queue_get(b2b_net* net, int32_t sid, int64_t* n, int32_t* offset, int32_t* pre,
                         int32_t* delay, int64_t cap) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(sid >= 0 && sid < (int)net->syns.size(), B2B_ERR_INVALID_ARG, "bad synapses %d", sid);
  CHECK(n != nullptr, B2B_ERR_INVALID_ARG, "n is NULL");
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  GUARD_BEGIN
  const Syn& sy = net->syns[sid];
  const Proj& pr = net->projs[sy.proj];
  const Group& gpre = net->groups[sy.pre_gid];
  const PopDev& S = net->pops[gpre.pop].dev;
  const int32_t nd = pr.dmax - pr.dmin + 1;
  CU(cudaStreamSynchronize(net->stream));
  const int64_t lo = gpre.offset + sy.pre_lo, hi = gpre.offset + sy.pre_hi;
  std::vector<int64_t> off((size_t)(hi - lo) * nd + 1);
  CU(cudaMemcpy(off.data(), pr.off + lo * (int64_t)nd, 8 * off.size(), cudaMemcpyDeviceToHost));
  std::vector<int32_t> cnt(S.ring_len);
  CU(cudaMemcpy(cnt.data(), S.ring_cnt, 4 * S.ring_len, cudaMemcpyDeviceToHost));
  std::vector<std::vector<int32_t>> rows(S.ring_len);
  struct E { int32_t a, p, d; };
  std::vector<E> out;
  const int64_t last = net->ts - 1;
  for (int32_t a = 1; a <= pr.dmax && last >= 0; ++a) {
    for (int32_t d = std::max(a, pr.dmin); d <= pr.dmax; ++d) {
      const int64_t st = last + a - d;
      if (st < 0) continue;
      const int slot = (int)(st % S.ring_len);
      if (rows[slot].empty() && cnt[slot] > 0) {
        rows[slot].resize(cnt[slot]);
        CU(cudaMemcpy(rows[slot].data(), S.ring_idx + (int64_t)slot * S.n, 4 * (size_t)cnt[slot],
                      cudaMemcpyDeviceToHost));
      }
      for (int32_t x : rows[slot]) {
        if (x < lo || x >= hi) continue;
        const int64_t key = (int64_t)(x - lo) * nd + (d - pr.dmin);
        if (off[key + 1] > off[key]) out.push_back({a, (int32_t)(x - gpre.offset), d});
      }
    }
  }
  std::sort(out.begin(), out.end(), [](const E& x, const E& y) {
    if (x.a != y.a) return x.a < y.a;
    if (x.p != y.p) return x.p < y.p;
    return x.d < y.d;
  });
  *n = (int64_t)out.size();
  for (int64_t k = 0; k < (int64_t)out.size() && k < cap; ++k) {
    if (offset) offset[k] = out[k].a;
    if (pre) pre[k] = out[k].p;
    if (delay) delay[k] = out[k].d;
  }
  return B2B_OK;
  GUARD_END
}

b2b_status b2b_rng_uniforms_get(b2b_net* net, int32_t gid, void* host, int64_t steps,
                                int64_t n) {
  return rng_buffer_get(net, gid, false, host, steps, n);
}

b2b_status b2b_rng_normals_get(b2b_net* net, int32_t gid, void* host, int64_t steps,
                               int64_t n) {
  return rng_buffer_get(net, gid, true, host, steps, n);
}

b2b_status b2b_group_model(b2b_net* net, int64_t n, int32_t dtype, const char* module_path,
                           double refractory, int32_t* gid) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(module_path != nullptr, B2B_ERR_INVALID_ARG, "module_path is NULL");
  CHECK(refractory >= 0 && std::isfinite(refractory), B2B_ERR_INVALID_ARG, "bad refractory");
  GUARD_BEGIN
  // The object stays loaded until the process exits: its kernels may be referenced by
  // captured graphs and other nets.
  void* dl = dlopen(module_path, RTLD_NOW | RTLD_LOCAL);
  CHECK(dl != nullptr, B2B_ERR_INVALID_ARG, "cannot load model %s: %s", module_path, dlerror());
  auto info = reinterpret_cast<ModelInfoFn>(dlsym(dl, "b2b_model_info_v1"));
  auto launch = reinterpret_cast<ModelLaunchFn>(dlsym(dl, "b2b_model_launch_v1"));
  CHECK(info && launch, B2B_ERR_INVALID_ARG, "%s exports no b2b model entry points",
        module_path);
  Group g;
  g.kind = KIND_MODEL; g.n = n; g.dtype = dtype;
  CHECK(info(&g.minfo) == 0 && g.minfo.abi == B2B_MODEL_ABI, B2B_ERR_UNSUPPORTED,
        "model %s: ABI %d, this library expects %d", module_path, g.minfo.abi, B2B_MODEL_ABI);
  CHECK(g.minfo.n_vars >= 1 && g.minfo.n_vars <= B2B_MODEL_MAX_VARS && g.minfo.n_normal >= 0 &&
            g.minfo.n_uniform >= 0, B2B_ERR_UNSUPPORTED, "model %s: bad shape", module_path);
  g.model_dl = dl;
  g.model_launch = launch;
  g.model_refractory = refractory;
  return add_group(net, std::move(g), gid);
  GUARD_END
}

b2b_status b2b_out_degree(b2b_net* net, int32_t gid, int32_t* host, int64_t n) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  CHECK(gid >= 0 && gid < (int32_t)net->groups.size() && host != nullptr, B2B_ERR_INVALID_ARG,
        "bad arguments");
  const Group& g = net->groups[gid];
  CHECK(n == g.n, B2B_ERR_INVALID_ARG, "n must be the group size");
  GUARD_BEGIN
  int32_t* d = nullptr;
  CU(cudaMalloc(&d, sizeof(int32_t) * std::max<int64_t>(n, 1)));
  cudaError_t e = cudaMemsetAsync(d, 0, sizeof(int32_t) * n, net->stream);
  for (const Proj& pr : net->projs)
    if (e == cudaSuccess && pr.src_pop == g.pop && n > 0 && pr.retire_after < 0)
      e = add_out_degree(pr.off, pr.dev.nd, g.offset, n, d, net->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(host, d, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, net->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(net->stream);
  cudaFree(d);
  CU(e);
  return B2B_OK;
  GUARD_END
}

b2b_status b2b_syn_set_delays(b2b_net* net, int32_t sid, const int32_t* delay_steps,
                              int64_t n) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  CHECK(sid >= 0 && sid < (int)net->syns.size(), B2B_ERR_INVALID_ARG, "bad synapses id %d", sid);
  Syn& sy = net->syns[sid];
  CHECK(!sy.generated, B2B_ERR_UNSUPPORTED,
        "delays of connectivity generated on the GPU are fixed");
  CHECK(sy.effect == B2B_EFFECT_ADD, B2B_ERR_UNSUPPORTED, "delays of STDP synapses are fixed");
  CHECK(!(net->cfg.flags & B2B_NET_SMALL), B2B_ERR_UNSUPPORTED,
        "B2B_NET_SMALL keeps the small-network path, whose delays are fixed");
  CHECK(delay_steps && n == sy.n, B2B_ERR_INVALID_ARG, "n must be the synapse count");
  for (int64_t k = 0; k < n; ++k)
    CHECK(delay_steps[k] >= 0, B2B_ERR_INVALID_ARG, "negative delay at synapse %lld",
          (long long)k);
  // the small-network path, if the autotuner chose it, hands over to the per-step kernels
  // (its connectivity views are built once)
  if (net->small_ok) {
    net->small = false;
    net->small_ok = false;
    if (net->graph) {
      cudaGraphExecDestroy(net->graph);
      net->graph = nullptr;
    }
  }
  GUARD_BEGIN
  CU(cudaStreamSynchronize(net->stream));
  if (net->graph) {
    cudaGraphExecDestroy(net->graph);
    net->graph = nullptr;
  }
  const int64_t T = net->ts;                  // spikes from this step on use the new delays
  const int pj = sy.proj;
  // the projection as built keeps delivering the spikes sent before step T
  Proj old = net->projs[pj];
  old.dev.src_hi = std::min(old.dev.src_hi, T);
  old.retire_after = T - 1 + old.dmax;
  // the new delays, and the projection rebuilt from its members
  sy.delay.assign(delay_steps, delay_steps + n);
  sy.dmin = n ? *std::min_element(sy.delay.begin(), sy.delay.end()) : sy.delay_scalar;
  sy.dmax = n ? *std::max_element(sy.delay.begin(), sy.delay.end()) : sy.delay_scalar;
  {
    Proj& pr = net->projs[pj];
    pr.allocs.clear();
    pr.dev = ProjDev{};
    pr.off = nullptr;
    pr.post = nullptr;
    pr.w = nullptr;
    pr.n_syn = 0;
    pr.max_bundle = 0;
    pr.dmin = INT32_MAX;
    pr.dmax = 0;
    for (int m : pr.members) {
      pr.dmin = std::min(pr.dmin, net->syns[m].dmin);
      pr.dmax = std::max(pr.dmax, net->syns[m].dmax);
    }
    Pop& src = net->pops[pr.src_pop];
    if (pr.dmax + 2 > src.dev.ring_len) {
      if (b2b_status st = grow_ring(net, pr.src_pop, pr.dmax + 2)) return st;
      old.dev.src_ring_idx = src.dev.ring_idx;
      old.dev.src_ring_cnt = src.dev.ring_cnt;
      old.dev.src_ring_len = src.dev.ring_len;
    }
    if (b2b_status st = build_proj(net, pj)) return st;
    net->projs[pj].dev.src_lo = T;
  }
  if (old.dev.src_lo < old.dev.src_hi && old.retire_after >= T) {
    net->projs.push_back(std::move(old));
  } else {
    for (void* a : old.allocs) cudaFree(a);
  }
  build_add_batches(net);
  refresh_two_launch(net);
  return B2B_OK;
  GUARD_END
}

b2b_status b2b_syn_count(b2b_net* net, int32_t sid, int64_t* n) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(sid >= 0 && sid < (int)net->syns.size() && n, B2B_ERR_INVALID_ARG, "bad synapses %d",
        sid);
  CHECK(net->finalized || !net->syns[sid].generated, B2B_ERR_STATE,
        "generated synapses exist only after b2b_finalize");
  *n = net->syns[sid].n;
  return B2B_OK;
}

b2b_status b2b_syn_get(b2b_net* net, int32_t sid, int32_t var, void* host, int64_t n) {
  if (b2b_status st = check_net(net)) return st;
  CHECK(sid >= 0 && sid < (int)net->syns.size(), B2B_ERR_INVALID_ARG, "bad synapses %d", sid);
  CHECK(net->finalized, B2B_ERR_STATE, "call b2b_finalize first");
  const Syn& sy = net->syns[sid];
  CHECK(host && n == sy.n, B2B_ERR_INVALID_ARG, "expected %lld values", (long long)sy.n);
  CHECK(var >= B2B_SYN_I && var <= B2B_SYN_LASTUPDATE, B2B_ERR_INVALID_ARG, "bad variable %d",
        var);
  const Proj& pr = net->projs[sy.proj];
  CHECK(var <= B2B_SYN_W || pr.effect == B2B_EFFECT_STDP, B2B_ERR_INVALID_ARG,
        "variable %d exists only for STDP synapses", var);
  if (n == 0) return B2B_OK;
  const Group& gpre = net->groups[sy.pre_gid];
  const Group& gpost = net->groups[sy.post_gid];
  const int32_t nd = pr.dmax - pr.dmin + 1;
  const void* arr = nullptr;
  int64_t stride = 1;
  if (pr.effect == B2B_EFFECT_STDP && var >= B2B_SYN_W) {
    // component (var - W) of the interleaved {w, Apre, Apost, lastupdate} records
    arr = static_cast<const uint8_t*>(pr.dev.syn4) + real_size(pr.dtype) * (var - B2B_SYN_W);
    stride = 4;
  } else if (var == B2B_SYN_W) {
    arr = pr.w;
  }
  const int64_t* inv = sy.inv;  // NULL for generated synapses: positions are the numbering
  const size_t es = (var <= B2B_SYN_DELAY) ? 4 : real_size(pr.dtype);
  void* d_out = nullptr;
  CU(cudaMalloc(&d_out, es * n));
  cudaError_t e = gather_syn_var(pr, var, inv, sy.base, n,
                                 (gpre.offset + sy.pre_lo) * (int64_t)nd,
                                 (gpre.offset + sy.pre_hi) * (int64_t)nd, gpre.offset,
                                 gpost.offset, arr, stride, sy.w_scalar, d_out, net->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(host, d_out, es * n, cudaMemcpyDeviceToHost, net->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(net->stream);
  cudaFree(d_out);
  if (e != cudaSuccess) return fail(net, B2B_ERR_CUDA, "syn_get: %s", cudaGetErrorString(e));
  return B2B_OK;
}

}  // extern "C"
