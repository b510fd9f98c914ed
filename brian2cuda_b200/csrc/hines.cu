// Batched Hines solver for multicompartment (SpatialNeuron) HH neurons.
//
// Reference: brian2cuda/templates/spatialstateupdate.cu runs, per SpatialNeuron and step,
// five launches: channel update (108-113), `_tridiagsolve<<<branches, 1>>>` (128-192,
// Thomas algorithm with three right-hand sides per section), `_coupling<<<1, 1>>>` (202-307,
// the Hines elimination over the section tree on a single thread), `_combine<<<branches,
// 1>>>` (316-351) and `_currents` (359-387).  One neuron is one code object, so a batch of
// neurons costs five launches per neuron per step.
//
// Here one CTA owns one neuron and keeps its whole morphology (matrix diagonals, state,
// per-section and per-node arrays) in shared memory across a chunk of steps; the only
// global traffic inside the chunk is the soma spike count.  Per step: compartment-parallel
// channels, section-parallel Thomas solves, node-parallel assembly of the coupling system,
// then elimination and substitution level by level over the section tree (nodes of equal
// depth are independent), and a compartment-parallel combine.  The arithmetic of each
// step follows the reference's formulas term by term.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "kernels_common.cuh"

namespace b2b {
namespace {

constexpr int kHinesBlock = 256;
constexpr int kHinesMaxStepsPerLaunch = 1000;

struct HinesDev {
  int32_t n_neurons;
  int32_t nc_max, ns_max, nlev_max;
  const int64_t* comp_off;
  const int32_t* sec_off;
  const int32_t* lvl_base;
  const double *ab0, *ab1, *ab2;
  const int32_t* sec_of_comp;
  const int32_t *sec_start, *sec_end, *sec_pnode;
  const double *invr0, *invrn, *bplus, *bminus;
  const int32_t* child_off;   // per node (global node index = sec_off[b] + b + i), global edges
  const int32_t* child_sec;   // neuron-local section index per edge
  const int32_t* level_order; // per node slot: neuron-local node ids sorted by depth
  const int32_t* level_off;   // per neuron at lvl_base[b]: nlev+1 offsets into level_order
  double* v;
  void *m, *h, *n;
  double* Ic;
  const double* soma_I;       // per neuron injected current / soma area (A/m^2)
  int32_t* spikes;
  int32_t* above;
  double Cm, dt, El, EK, ENa, gl, gNa, gK, Vthr;
};

template <typename RC>
__device__ __forceinline__ RC hh_expeuler(RC x, RC a, RC b, RC dt) {
  const RC A = -(a + b);
  const RC BA = a / A;
  return -BA + (BA + x) * dexp(A * dt);
}

// Hodgkin-Huxley 1952 rates (examples/compartmental/hh_with_spikes_cuda.py:41-46), v in
// volts measured from rest, rates in 1/s; x/(exp(x/a) - 1) forms through z_over_expm1.
template <typename RC>
__device__ __forceinline__ void hh_gates(RC v, RC dt, RC& m, RC& h, RC& n) {
  const RC am = (RC)1000 * z_over_expm1(((RC)25e-3 - v) / (RC)10e-3);
  const RC bm = (RC)4000 * dexp(-v / (RC)18e-3);
  const RC ah = (RC)70 * dexp(-v / (RC)20e-3);
  const RC bh = (RC)1000 / (dexp(((RC)30e-3 - v) / (RC)10e-3) + (RC)1);
  const RC an = (RC)100 * z_over_expm1(((RC)10e-3 - v) / (RC)10e-3);
  const RC bn = (RC)125 * dexp(-v / (RC)80e-3);
  m = hh_expeuler(m, am, bm, dt);
  h = hh_expeuler(h, ah, bh, dt);
  n = hh_expeuler(n, an, bn, dt);
}

template <typename RC>
__global__ void __launch_bounds__(kHinesBlock)
hines_kernel(HinesDev H, int n_steps, int write_currents) {
  extern __shared__ __align__(16) uint8_t sm[];
  const int b = blockIdx.x;
  const int tid = threadIdx.x, bs = blockDim.x;
  const int64_t c0 = H.comp_off[b];
  const int nc = (int)(H.comp_off[b + 1] - c0);
  const int s0 = H.sec_off[b];
  const int ns = H.sec_off[b + 1] - s0;
  const int nB = ns + 1;
  const int nb0 = s0 + b;
  const int l0 = H.lvl_base[b];
  const int nlev = H.lvl_base[b + 1] - l0 - 1;
  const int NC = H.nc_max, NS = H.ns_max, NB = H.ns_max + 1;

  double* V = reinterpret_cast<double*>(sm);
  double* RHS = V + NC;
  double* UP = RHS + NC;
  double* UM = UP + NC;
  double* C = UM + NC;
  double* DIAG = C + NC;
  double* AB0 = DIAG + NC;
  double* AB1 = AB0 + NC;
  double* AB2 = AB1 + NC;
  double* PD = AB2 + NC;
  double* PP = PD + NB;
  double* BB = PP + NB;
  double* PCH = BB + NB;
  double* INVR0 = PCH + NS;
  double* INVRN = INVR0 + NS;
  double* BPL = INVRN + NS;
  double* BMI = BPL + NS;
  RC* M = reinterpret_cast<RC*>(BMI + NS);
  RC* Hh = M + NC;
  RC* N = Hh + NC;
  int32_t* SOC = reinterpret_cast<int32_t*>(N + NC);
  int32_t* SST = SOC + NC;
  int32_t* SEN = SST + NS;
  int32_t* SPN = SEN + NS;
  int32_t* COFF = SPN + NS;
  int32_t* CSEC = COFF + NB + 1;
  int32_t* LORD = CSEC + NS;
  int32_t* LOFF = LORD + NB;

  const RC* gm = static_cast<const RC*>(H.m);
  const RC* gh = static_cast<const RC*>(H.h);
  const RC* gn = static_cast<const RC*>(H.n);
  for (int j = tid; j < nc; j += bs) {
    V[j] = H.v[c0 + j];
    AB0[j] = H.ab0[c0 + j];
    AB1[j] = H.ab1[c0 + j];
    AB2[j] = H.ab2[c0 + j];
    M[j] = gm[c0 + j];
    Hh[j] = gh[c0 + j];
    N[j] = gn[c0 + j];
    SOC[j] = H.sec_of_comp[c0 + j];
  }
  for (int s = tid; s < ns; s += bs) {
    SST[s] = H.sec_start[s0 + s];
    SEN[s] = H.sec_end[s0 + s];
    SPN[s] = H.sec_pnode[s0 + s];
    INVR0[s] = H.invr0[s0 + s];
    INVRN[s] = H.invrn[s0 + s];
    BPL[s] = H.bplus[s0 + s];
    BMI[s] = H.bminus[s0 + s];
  }
  const int e0 = H.child_off[nb0];
  for (int i = tid; i <= nB; i += bs) COFF[i] = H.child_off[nb0 + i] - e0;
  for (int e = tid; e < ns; e += bs) CSEC[e] = H.child_sec[e0 + e];
  for (int k = tid; k < nB; k += bs) LORD[k] = H.level_order[nb0 + k];
  for (int L = tid; L <= nlev; L += bs) LOFF[L] = H.level_off[l0 + L];
  __syncthreads();

  const double cdt = H.Cm / H.dt;
  const double Isoma = H.soma_I[b];
  const RC dtR = (RC)H.dt;
  int above = H.above[b];
  int spikes = 0;

  for (int step = 0; step < n_steps; ++step) {
    // (1) channels: conductance and current at the start of the step, then the gates
    for (int j = tid; j < nc; j += bs) {
      const double v = V[j];
      RC m = M[j], h = Hh[j], n = N[j];
      const double md = (double)m, hd = (double)h, nd = (double)n;
      const double gna = H.gNa * (md * md * md * hd);
      const double gk = H.gK * (nd * nd * nd * nd);
      const double gtot = H.gl + gna + gk;
      double I0 = H.gl * H.El + gna * H.ENa + gk * H.EK;
      if (j == 0) I0 += Isoma;
      DIAG[j] = AB1[j] - gtot;
      RHS[j] = -cdt * v - I0;
      hh_gates<RC>((RC)v, dtR, m, h, n);
      M[j] = m;
      Hh[j] = h;
      N[j] = n;
    }
    __syncthreads();
    // (2) Thomas solve of each section for v*, u+ and u-
    for (int s = tid; s < ns; s += bs) {
      const int j0 = SST[s], j1 = SEN[s];
      for (int j = j0; j < j1; ++j) {
        const double bi = DIAG[j];
        const double cj = (j + 1 < j1) ? AB0[j + 1] : 0.0;
        const double vs = RHS[j];
        const double upj = (j == j1 - 1) ? BPL[s] : 0.0;
        const double umj = (j == j0) ? BMI[s] : 0.0;
        if (j == 0) {
          C[j] = cj / bi; RHS[j] = vs / bi; UP[j] = upj / bi; UM[j] = umj / bi;
        } else if (j == j0) {
          const double mm = 1.0 / bi;
          C[j] = cj * mm; RHS[j] = vs * mm; UP[j] = upj * mm; UM[j] = umj * mm;
        } else {
          const double ai = AB2[j - 1];
          const double mm = 1.0 / (bi - ai * C[j - 1]);
          C[j] = cj * mm;
          RHS[j] = (vs - ai * RHS[j - 1]) * mm;
          UP[j] = (upj - ai * UP[j - 1]) * mm;
          UM[j] = (umj - ai * UM[j - 1]) * mm;
        }
      }
      for (int j = j1 - 2; j >= j0; --j) {
        RHS[j] = RHS[j] - C[j] * RHS[j + 1];
        UP[j] = UP[j] - C[j] * UP[j + 1];
        UM[j] = UM[j] - C[j] * UM[j + 1];
      }
    }
    __syncthreads();
    // (3) coupling system, one row per node
    for (int i = tid; i < nB; i += bs) {
      double pd, bb;
      if (i == 0) {
        const int f = SST[0];
        pd = UM[f] - 1.0;
        bb = -RHS[f];
        PCH[COFF[0]] = UP[f];
      } else {
        const int s = i - 1;
        const int last = SEN[s] - 1;
        pd = (1.0 - UP[last]) * INVRN[s];
        PP[s] = -UM[last] * INVRN[s];
        bb = RHS[last] * INVRN[s];
        for (int e = COFF[i]; e < COFF[i + 1]; ++e) {
          const int cs = CSEC[e];
          const int f = SST[cs];
          pd += (1.0 - UM[f]) * INVR0[cs];
          PCH[e] = -UP[f] * INVR0[cs];
          bb += RHS[f] * INVR0[cs];
        }
      }
      PD[i] = pd;
      BB[i] = bb;
    }
    __syncthreads();
    // (4) elimination, deepest level first
    for (int L = nlev - 1; L >= 0; --L) {
      for (int k = LOFF[L] + tid; k < LOFF[L + 1]; k += bs) {
        const int i = LORD[k];
        double pd = PD[i], bb = BB[i];
        for (int e = COFF[i]; e < COFF[i + 1]; ++e) {
          const int j = CSEC[e] + 1;
          const double sub = PCH[e] / PD[j];
          pd = pd - sub * PP[j - 1];
          bb = bb - sub * BB[j];
        }
        PD[i] = pd;
        BB[i] = bb;
      }
      __syncthreads();
    }
    // (5) substitution, root first
    if (tid == 0) BB[0] = BB[0] / PD[0];
    __syncthreads();
    for (int L = 1; L < nlev; ++L) {
      for (int k = LOFF[L] + tid; k < LOFF[L + 1]; k += bs) {
        const int i = LORD[k];
        const int j = SPN[i - 1];
        BB[i] = (BB[i] - PP[i - 1] * BB[j]) / PD[i];
      }
      __syncthreads();
    }
    // (6) combine the particular and homogeneous solutions; capacitive current
    const bool last_step = step == n_steps - 1;
    for (int j = tid; j < nc; j += bs) {
      const int s = SOC[j];
      const double vn = RHS[j] + BB[SPN[s]] * UM[j] + BB[s + 1] * UP[j];
      if (last_step && write_currents) H.Ic[c0 + j] = H.Cm * (vn - V[j]) / H.dt;
      V[j] = vn;
    }
    __syncthreads();
    if (tid == 0) {
      const int ab = V[0] > H.Vthr ? 1 : 0;
      if (ab && !above) ++spikes;
      above = ab;
    }
  }
  RC* wm = static_cast<RC*>(H.m);
  RC* wh = static_cast<RC*>(H.h);
  RC* wn = static_cast<RC*>(H.n);
  for (int j = tid; j < nc; j += bs) {
    H.v[c0 + j] = V[j];
    wm[c0 + j] = M[j];
    wh[c0 + j] = Hh[j];
    wn[c0 + j] = N[j];
  }
  if (tid == 0) {
    H.spikes[b] += spikes;
    H.above[b] = above;
  }
}

size_t hines_smem(int nc, int ns, int nlev, int rc_size) {
  const size_t NB = (size_t)ns + 1;
  return sizeof(double) * (9 * (size_t)nc + 3 * NB + 5 * (size_t)ns) + rc_size * 3 * (size_t)nc +
         sizeof(int32_t) * ((size_t)nc + 4 * (size_t)ns + NB + 1 + NB + (size_t)nlev + 1);
}

}  // namespace
}  // namespace b2b

struct b2b_hines {
  b2b_net* net = nullptr;
  b2b::HinesDev dev{};
  int channel_dtype = B2B_F32;
  int64_t n_comp = 0;
  int32_t n_neurons = 0;
  size_t smem = 0;
  std::vector<double> soma_area;
  std::vector<void*> allocs;
  std::string err;
};

using namespace b2b;

namespace {

template <typename T>
cudaError_t upload(b2b_hines* h, const T** dst, const std::vector<T>& src) {
  T* d = nullptr;
  cudaError_t e = cudaMalloc((void**)&d, sizeof(T) * std::max<size_t>(src.size(), 1));
  if (e != cudaSuccess) return e;
  h->allocs.push_back(d);
  if (!src.empty()) e = cudaMemcpy(d, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice);
  *dst = d;
  return e;
}

}  // namespace

extern "C" {

b2b_status b2b_hines_create(b2b_net* net, int32_t n_neurons, const int64_t* comp_off,
                            const int32_t* sec_off, const int32_t* sec_start,
                            const int32_t* sec_end, const int32_t* sec_parent,
                            const double* diameter, const double* length,
                            const b2b_hines_params* p, b2b_hines** out) {
  if (!net || !out || !p || n_neurons <= 0 || !comp_off || !sec_off || !sec_start || !sec_end ||
      !sec_parent || !diameter || !length)
    return B2B_ERR_INVALID_ARG;
  if (p->channel_dtype != B2B_F32 && p->channel_dtype != B2B_F64) return B2B_ERR_INVALID_ARG;
  if (!(p->Cm > 0) || !(p->Ri > 0)) return B2B_ERR_INVALID_ARG;
  if (cudaSetDevice(net->cfg.device) != cudaSuccess) return B2B_ERR_CUDA;
  *out = nullptr;
  const double dt = net->cfg.dt;
  try {
    if (comp_off[0] != 0 || sec_off[0] != 0) return B2B_ERR_INVALID_ARG;
    const int64_t n_comp = comp_off[n_neurons];
    const int32_t n_sec = sec_off[n_neurons];
    std::vector<double> ab0(n_comp, 0.0), ab1(n_comp, 0.0), ab2(n_comp, 0.0);
    std::vector<int32_t> soc(n_comp), sst(n_sec), sen(n_sec), spn(n_sec);
    std::vector<double> invr0(n_sec), invrn(n_sec), bpl(n_sec), bmi(n_sec);
    std::vector<int32_t> child_off, child_sec, level_order, level_off, lvl_base;
    std::vector<double> area(n_comp), rl(n_comp), invr(n_comp, 0.0);
    std::vector<double> soma_area(n_neurons);
    int nc_max = 0, ns_max = 0, nlev_max = 0;
    const double Ri = p->Ri, Cm = p->Cm;
    for (int b = 0; b < n_neurons; ++b) {
      const int64_t c0 = comp_off[b], c1 = comp_off[b + 1];
      const int s0 = sec_off[b], s1 = sec_off[b + 1];
      const int nc = (int)(c1 - c0), ns = s1 - s0;
      if (nc <= 0 || ns <= 0 || nc > (1 << 20)) return B2B_ERR_INVALID_ARG;
      nc_max = std::max(nc_max, nc);
      ns_max = std::max(ns_max, ns);
      // morphology checks: sections contiguous, in topological order, root first
      if (sec_start[s0] != 0 || sec_parent[s0] != -1 || sec_end[s1 - 1] != nc)
        return B2B_ERR_INVALID_ARG;
      for (int s = 0; s < ns; ++s) {
        if (sec_end[s0 + s] <= sec_start[s0 + s]) return B2B_ERR_INVALID_ARG;
        if (s > 0 && sec_start[s0 + s] != sec_end[s0 + s - 1]) return B2B_ERR_INVALID_ARG;
        if (s > 0 && (sec_parent[s0 + s] < 0 || sec_parent[s0 + s] >= s)) return B2B_ERR_INVALID_ARG;
      }
      for (int64_t c = c0; c < c1; ++c) {
        if (!(diameter[c] > 0) || !(length[c] > 0)) return B2B_ERR_INVALID_ARG;
        area[c] = M_PI * diameter[c] * length[c];
        rl[c] = M_PI * diameter[c] * diameter[c] / (2.0 * length[c]);
      }
      soma_area[b] = area[c0];
      // matrix (brian2cuda/templates/spatialstateupdate.cu:36-77, neuron-local indices)
      for (int64_t c = c0 + 1; c < c1; ++c) invr[c] = 1.0 / (Ri * (1.0 / rl[c - 1] + 1.0 / rl[c]));
      for (int s = 0; s < ns; ++s) invr[c0 + sec_start[s0 + s]] = 0.0;
      for (int64_t c = c0; c < c1; ++c) ab1[c] = (-(Cm / dt) - invr[c] / area[c]);
      for (int64_t c = c0 + 1; c < c1; ++c) {
        ab0[c] = invr[c] / area[c - 1];
        ab2[c - 1] = invr[c] / area[c];
        ab1[c - 1] -= invr[c] / area[c - 1];
      }
      for (int s = 0; s < ns; ++s) {
        const int64_t first = c0 + sec_start[s0 + s];
        const int64_t last = c0 + sec_end[s0 + s] - 1;
        const double i0 = rl[first] / Ri, in = rl[last] / Ri;
        invr0[s0 + s] = i0;
        invrn[s0 + s] = in;
        ab1[first] -= (i0 / area[first]);
        ab1[last] -= (in / area[last]);
        bpl[s0 + s] = -(in / area[last]);
        bmi[s0 + s] = -(i0 / area[first]);
        sst[s0 + s] = sec_start[s0 + s];
        sen[s0 + s] = sec_end[s0 + s];
        spn[s0 + s] = s == 0 ? 0 : sec_parent[s0 + s] + 1;
        for (int64_t c = first; c <= last; ++c) soc[c] = s;
      }
      // nodes: node 0 = sealed start of the root, node s+1 = end of section s
      const int nB = ns + 1;
      std::vector<std::vector<int>> kids(nB);
      kids[0].push_back(0);
      for (int s = 1; s < ns; ++s) kids[spn[s0 + s]].push_back(s);
      std::vector<int> depth(nB, 0);
      for (int s = 0; s < ns; ++s) depth[s + 1] = depth[spn[s0 + s]] + 1;
      const int nlev = *std::max_element(depth.begin(), depth.end()) + 1;
      nlev_max = std::max(nlev_max, nlev);
      const int edge_base = (int)child_sec.size();
      for (int i = 0; i < nB; ++i) {
        child_off.push_back((int)child_sec.size());
        for (int s : kids[i]) child_sec.push_back(s);
      }
      (void)edge_base;
      std::vector<int> order(nB);
      for (int i = 0; i < nB; ++i) order[i] = i;
      std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return depth[a] < depth[c]; });
      lvl_base.push_back((int)level_off.size());
      for (int i = 0; i < nB; ++i) level_order.push_back(order[i]);
      int k = 0;
      for (int L = 0; L <= nlev; ++L) {
        while (k < nB && depth[order[k]] < L) ++k;
        level_off.push_back(k);
      }
    }
    child_off.push_back((int)child_sec.size());
    lvl_base.push_back((int)level_off.size());

    const int rc = p->channel_dtype == B2B_F32 ? 4 : 8;
    const size_t smem = hines_smem(nc_max, ns_max, nlev_max, rc);
    int dev_smem = 0;
    cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, net->cfg.device);
    if ((int64_t)smem > dev_smem) return B2B_ERR_UNSUPPORTED;

    b2b_hines* h = new b2b_hines();
    h->net = net;
    h->channel_dtype = p->channel_dtype;
    h->n_comp = n_comp;
    h->n_neurons = n_neurons;
    h->smem = smem;
    h->soma_area = soma_area;
    HinesDev& D = h->dev;
    D.n_neurons = n_neurons;
    D.nc_max = nc_max;
    D.ns_max = ns_max;
    D.nlev_max = nlev_max;
    D.Cm = Cm; D.dt = dt; D.El = p->El; D.EK = p->EK; D.ENa = p->ENa; D.gl = p->gl;
    D.gNa = p->gNa; D.gK = p->gK; D.Vthr = p->Vthr;
    std::vector<int64_t> co(comp_off, comp_off + n_neurons + 1);
    std::vector<int32_t> so(sec_off, sec_off + n_neurons + 1);
    cudaError_t e = cudaSuccess;
    auto up = [&](auto** dst, const auto& src) {
      if (e == cudaSuccess) e = upload(h, dst, src);
    };
    up(&D.comp_off, co); up(&D.sec_off, so); up(&D.lvl_base, lvl_base);
    up(&D.ab0, ab0); up(&D.ab1, ab1); up(&D.ab2, ab2); up(&D.sec_of_comp, soc);
    up(&D.sec_start, sst); up(&D.sec_end, sen); up(&D.sec_pnode, spn);
    up(&D.invr0, invr0); up(&D.invrn, invrn); up(&D.bplus, bpl); up(&D.bminus, bmi);
    up(&D.child_off, child_off); up(&D.child_sec, child_sec);
    up(&D.level_order, level_order); up(&D.level_off, level_off);
    std::vector<double> zeros_d(n_comp, 0.0), zero_I(n_neurons, 0.0);
    std::vector<int32_t> zeros_i(n_neurons, 0);
    const double* cv = nullptr;
    up(&cv, zeros_d); D.v = const_cast<double*>(cv);
    up(&cv, zeros_d); D.Ic = const_cast<double*>(cv);
    up(&D.soma_I, zero_I);
    const int32_t* ci = nullptr;
    up(&ci, zeros_i); D.spikes = const_cast<int32_t*>(ci);
    up(&ci, zeros_i); D.above = const_cast<int32_t*>(ci);
    for (void** g : {&D.m, &D.h, &D.n}) {
      if (e != cudaSuccess) break;
      e = cudaMalloc(g, rc * std::max<int64_t>(n_comp, 1));
      if (e == cudaSuccess) { h->allocs.push_back(*g); e = cudaMemset(*g, 0, rc * n_comp); }
    }
    if (e == cudaSuccess)
      e = rc == 4 ? cudaFuncSetAttribute(hines_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                  : cudaFuncSetAttribute(hines_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) {
      b2b_hines_destroy(h);
      return e == cudaErrorMemoryAllocation ? B2B_ERR_OOM : B2B_ERR_CUDA;
    }
    net->hines.push_back(h);
    *out = h;
    return B2B_OK;
  } catch (const std::bad_alloc&) {
    return B2B_ERR_OOM;
  }
}

b2b_status b2b_hines_set_current(b2b_hines* h, const double* soma_current) {
  if (!h) return B2B_ERR_INVALID_ARG;
  std::vector<double> I(h->n_neurons, 0.0);
  if (soma_current)
    for (int b = 0; b < h->n_neurons; ++b) I[b] = soma_current[b] / h->soma_area[b];
  cudaSetDevice(h->net->cfg.device);
  cudaError_t e = cudaMemcpy(const_cast<double*>(h->dev.soma_I), I.data(), 8 * I.size(),
                             cudaMemcpyHostToDevice);
  return e == cudaSuccess ? B2B_OK : B2B_ERR_CUDA;
}

static void* hines_var(b2b_hines* h, int32_t var, size_t* es) {
  const size_t rc = h->channel_dtype == B2B_F32 ? 4 : 8;
  switch (var) {
    case 0: *es = 8; return h->dev.v;
    case 1: *es = rc; return h->dev.m;
    case 2: *es = rc; return h->dev.h;
    case 3: *es = rc; return h->dev.n;
    case 4: *es = 8; return h->dev.Ic;
    default: return nullptr;
  }
}

b2b_status b2b_hines_state_set(b2b_hines* h, int32_t var, const void* host, int64_t n) {
  if (!h || !host || n != h->n_comp) return B2B_ERR_INVALID_ARG;
  size_t es = 0;
  void* d = hines_var(h, var, &es);
  if (!d) return B2B_ERR_INVALID_ARG;
  cudaSetDevice(h->net->cfg.device);
  cudaStreamSynchronize(h->net->stream);
  return cudaMemcpy(d, host, es * n, cudaMemcpyHostToDevice) == cudaSuccess ? B2B_OK : B2B_ERR_CUDA;
}

b2b_status b2b_hines_state_get(b2b_hines* h, int32_t var, void* host, int64_t n) {
  if (!h || !host || n != h->n_comp) return B2B_ERR_INVALID_ARG;
  size_t es = 0;
  void* d = hines_var(h, var, &es);
  if (!d) return B2B_ERR_INVALID_ARG;
  cudaSetDevice(h->net->cfg.device);
  cudaStreamSynchronize(h->net->stream);
  return cudaMemcpy(host, d, es * n, cudaMemcpyDeviceToHost) == cudaSuccess ? B2B_OK : B2B_ERR_CUDA;
}

b2b_status b2b_hines_run(b2b_hines* h, int64_t n_steps) {
  if (!h || n_steps < 0) return B2B_ERR_INVALID_ARG;
  cudaSetDevice(h->net->cfg.device);
  while (n_steps > 0) {
    const int k = (int)std::min<int64_t>(n_steps, kHinesMaxStepsPerLaunch);
    const int wc = n_steps == k ? 1 : 0;
    if (h->channel_dtype == B2B_F32)
      hines_kernel<float><<<h->n_neurons, kHinesBlock, h->smem, h->net->stream>>>(h->dev, k, wc);
    else
      hines_kernel<double><<<h->n_neurons, kHinesBlock, h->smem, h->net->stream>>>(h->dev, k, wc);
    if (cudaGetLastError() != cudaSuccess) return B2B_ERR_CUDA;
    h->net->launches += 1;
    n_steps -= k;
  }
  return B2B_OK;
}

b2b_status b2b_hines_spike_counts(b2b_hines* h, int32_t* host, int32_t n) {
  if (!h || !host || n != h->n_neurons) return B2B_ERR_INVALID_ARG;
  cudaSetDevice(h->net->cfg.device);
  cudaStreamSynchronize(h->net->stream);
  return cudaMemcpy(host, h->dev.spikes, 4 * (size_t)n, cudaMemcpyDeviceToHost) == cudaSuccess
             ? B2B_OK
             : B2B_ERR_CUDA;
}

b2b_status b2b_hines_destroy(b2b_hines* h) {
  if (!h) return B2B_ERR_INVALID_ARG;
  if (h->net) {
    cudaSetDevice(h->net->cfg.device);
    auto& v = h->net->hines;
    v.erase(std::remove(v.begin(), v.end(), h), v.end());
  }
  for (void* a : h->allocs) cudaFree(a);
  delete h;
  return B2B_OK;
}

}  // extern "C"
