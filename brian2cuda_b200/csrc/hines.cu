// Batched Hines solver for multicompartment (SpatialNeuron) HH neurons.
//
// Reference: brian2cuda/templates/spatialstateupdate.cu runs, per SpatialNeuron and step,
// five launches: channel update (108-113), `_tridiagsolve<<<branches, 1>>>` (128-192,
// Thomas algorithm with three right-hand sides per section), `_coupling<<<1, 1>>>` (202-307,
// the Hines elimination over the section tree on a single thread), `_combine<<<branches,
// 1>>>` (316-351) and `_currents` (359-387).  One neuron is one code object, so a batch of
// neurons costs five launches per neuron per step.
//
// The method (domain decomposition of the backward-Euler cable equation), restated from the
// mathematics: compartment j couples to compartment j-1 of its section through the axial
// conductance g[j] (0 at a section's first compartment), a section's first and last
// compartments to its start and end nodes through g0 and gn.  Per section, three
// tridiagonal solves with one matrix give x* (both node voltages 0) and the responses u_start,
// u_end to a unit voltage at either node, so that v = x* + V_start u_start + V_end u_end;
// Kirchhoff's current law at the nodes (node 0: the sealed start of the root section, node
// s+1: the end of section s) gives a tree-shaped system in the node voltages.
//
// Here one CTA owns one neuron and keeps its whole morphology (matrix rows, state,
// per-section and per-node arrays) in shared memory across a chunk of steps; the only
// global traffic inside the chunk is the soma spike count.  Per step: compartment-parallel
// channels, section-parallel tridiagonal solves, node-parallel assembly of the node
// equations, then elimination (each node pulls in its children) and substitution level by
// level over the section tree (nodes of equal depth are independent), and a
// compartment-parallel combination.
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
constexpr int kHinesLargeCtas = 3;   // CTAs per SM of the large class (shared-memory bound)
constexpr int kHinesSmallCtas = 5;   // and of the small class

struct HinesDev {
  int32_t n_neurons;
  int32_t nc_max, ns_max, nlev_max;
  const int64_t* comp_off;
  const int32_t* sec_off;
  const int32_t* lvl_base;
  // per compartment: matrix row without the membrane conductance (low couples j to j-1, up
  // couples j to j+1; both 0 across section boundaries)
  const double *low, *diag, *up;
  const int32_t* sec_of_comp;
  const int32_t *sec_start, *sec_end, *sec_pnode;
  // per section: node couplings, and the right-hand side of the unit-node solves at the
  // first (-g0/area) and last (-gn/area) compartment
  const double *g0, *gn, *rhs_first, *rhs_last;
  const int32_t* child_off;   // per node (global node index = sec_off[b] + b + i), global edges
  const int32_t* child_sec;   // neuron-local section index per edge
  // per node slot, nodes sorted by depth: {node, parent node (-1 for node 0), first child
  // edge, end of its child edges} (neuron-local), 4 ints
  const int32_t* level_rec;
  const int32_t* level_off;   // per neuron at lvl_base[b]: nlev+1 offsets into level_rec
  double* v;
  void *m, *h, *n;
  double* Ic;
  const double* soma_I;       // per neuron injected current / soma area (A/m^2)
  int32_t* spikes;
  int32_t* above;
  double Cm, dt, El, EK, ENa, gl, gNa, gK, Vthr;
  // neuron of CTA k: neurons by decreasing estimated cost, so that the CTAs the block
  // scheduler starts last (when fewer than all neurons fit on the GPU at once) are the
  // shortest
  const int32_t* order;
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

// 1/x for a finite, normal, nonzero x: the reciprocal unit's approximation refined by two
// Newton-Raphson steps (y <- y + y (1 - x y), each step doubling the correct bits), within
// an ulp or two of the correctly rounded quotient.  The solver's serial chains (the pivots of
// a section, the node system level by level) take one reciprocal per link; the IEEE
// division's longer sequence made them several times longer.
__device__ __forceinline__ double recip(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}

// MINB: CTAs per SM the register budget is sized for.  The large class runs 3 per SM (its
// shared memory allows no more), so its kernel may keep its values in 80 registers instead of
// spilling; the small class runs 5 per SM.
template <typename RC, int MINB>
__global__ void __launch_bounds__(kHinesBlock, MINB)
hines_kernel(HinesDev H, int n_steps, int write_currents) {
  extern __shared__ __align__(16) uint8_t sm[];
  const int b = H.order[blockIdx.x];
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

  int4* REC = reinterpret_cast<int4*>(sm);   // level records, first (16-byte aligned)
  // The constant matrix rows (low, diag, up) and the compartment-to-section map are read
  // through the read-only cache rather than kept here, so that three CTAs fit an SM and one
  // neuron's serial phases overlap other neurons' parallel ones.
  double* V = reinterpret_cast<double*>(REC + NB);
  double* X = V + NC;          // x*, first the right-hand side of the membrane solve
  double* UE = X + NC;         // u_end
  double* US = UE + NC;        // u_start
  double* DG = US + NC;        // diagonal with the membrane conductance of the step, then
                               // the eliminated super-diagonal
  double* DN = DG + NC;        // node equations: diagonal,
  double* TOWARD = DN + NB;    // coefficient of the parent node (node >= 1),
  double* RHSN = TOWARD + NB;  // right-hand side,
  double* INTO = RHSN + NB;    // per node >= 1: its coefficient in its parent's equation
  double* INV = INTO + NB;     // 1 / final diagonal, per node
  double* G0 = INV + NB;
  double* GN = G0 + NS;
  double* RF = GN + NS;
  double* RL = RF + NS;
  RC* M = reinterpret_cast<RC*>(RL + NS);
  RC* Hh = M + NC;
  RC* N = Hh + NC;
  int32_t* SST = reinterpret_cast<int32_t*>(N + NC);
  int32_t* SEN = SST + NS;
  int32_t* SPN = SEN + NS;
  int32_t* COFF = SPN + NS;
  int32_t* CSEC = COFF + NB + 1;
  int32_t* LOFF = CSEC + NS;

  const RC* gm = static_cast<const RC*>(H.m);
  const RC* gh = static_cast<const RC*>(H.h);
  const RC* gn = static_cast<const RC*>(H.n);
  for (int j = tid; j < nc; j += bs) {
    V[j] = H.v[c0 + j];
    M[j] = gm[c0 + j];
    Hh[j] = gh[c0 + j];
    N[j] = gn[c0 + j];
  }
  for (int s = tid; s < ns; s += bs) {
    SST[s] = H.sec_start[s0 + s];
    SEN[s] = H.sec_end[s0 + s];
    SPN[s] = H.sec_pnode[s0 + s];
    G0[s] = H.g0[s0 + s];
    GN[s] = H.gn[s0 + s];
    RF[s] = H.rhs_first[s0 + s];
    RL[s] = H.rhs_last[s0 + s];
  }
  const int e0 = H.child_off[nb0];
  for (int i = tid; i <= nB; i += bs) COFF[i] = H.child_off[nb0 + i] - e0;
  for (int e = tid; e < ns; e += bs) CSEC[e] = H.child_sec[e0 + e];
  for (int k = tid; k < nB; k += bs)
    REC[k] = make_int4(H.level_rec[4 * (nb0 + k)], H.level_rec[4 * (nb0 + k) + 1],
                       H.level_rec[4 * (nb0 + k) + 2], H.level_rec[4 * (nb0 + k) + 3]);
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
      DG[j] = __ldg(H.diag + c0 + j) - gtot;
      X[j] = -cdt * v - I0;
      hh_gates<RC>((RC)v, dtR, m, h, n);
      M[j] = m;
      Hh[j] = h;
      N[j] = n;
    }
    __syncthreads();
    // (2) per section, one pass of forward elimination (reciprocal pivot) and back
    // substitution for the three right-hand sides
    for (int s = tid; s < ns; s += bs) {
      const int j0 = SST[s], j1 = SEN[s];
      double cprev = 0.0, xprev = 0.0, sprev = 0.0, eprev = 0.0;
      for (int j = j0; j < j1; ++j) {
        const double lw = j > j0 ? __ldg(H.low + c0 + j) : 0.0;
        const double piv = recip(DG[j] - lw * cprev);
        cprev = __ldg(H.up + c0 + j) * piv;
        DG[j] = cprev;   // the diagonal is not needed again
        X[j] = (X[j] - lw * xprev) * piv;
        US[j] = ((j == j0 ? RF[s] : 0.0) - lw * sprev) * piv;
        UE[j] = ((j == j1 - 1 ? RL[s] : 0.0) - lw * eprev) * piv;
        xprev = X[j];
        sprev = US[j];
        eprev = UE[j];
      }
      for (int j = j1 - 2; j >= j0; --j) {
        X[j] -= DG[j] * X[j + 1];
        US[j] -= DG[j] * US[j + 1];
        UE[j] -= DG[j] * UE[j + 1];
      }
    }
    __syncthreads();
    // (3) node equations: node i's current balance in its own voltage (DN), its parent
    // node's (TOWARD) and its children's end nodes' (INTO, stored with the child node)
    for (int i = tid; i < nB; i += bs) {
      double dn, rh;
      if (i == 0) {
        // the root's start takes the voltage of the root's first compartment
        const int f = SST[0];
        dn = US[f] - 1.0;
        rh = -X[f];
        INTO[1] = UE[f];
      } else {
        const int s = i - 1;
        const int l = SEN[s] - 1;
        dn = GN[s] * (1.0 - UE[l]);
        TOWARD[i] = -GN[s] * US[l];
        rh = GN[s] * X[l];
        for (int e = COFF[i]; e < COFF[i + 1]; ++e) {
          const int cs = CSEC[e];
          const int f = SST[cs];
          dn += G0[cs] * (1.0 - US[f]);
          INTO[cs + 1] = -G0[cs] * UE[f];
          rh += G0[cs] * X[f];
        }
      }
      DN[i] = dn;
      RHSN[i] = rh;
    }
    __syncthreads();
    // (4)-(5) the node system on the first warp alone, level by level with warp barriers (a
    // level holds few nodes; CTA-wide barriers per level would idle every other warp)
    if (tid < 32) {
      // (4) elimination, deepest level first: each node takes in its children's equations;
      // a record gives the node and its child edges at once, and children are taken in
      // pairs so that their loads and divisions overlap (the order of the updates is the
      // children's order)
      for (int L = nlev - 1; L >= 0; --L) {
        for (int k = LOFF[L] + tid; k < LOFF[L + 1]; k += 32) {
          const int4 r = REC[k];
          double dn = DN[r.x], rh = RHSN[r.x];
          int e = r.z;
          for (; e + 1 < r.w; e += 2) {
            const int ca = CSEC[e] + 1, cb = CSEC[e + 1] + 1;   // the children's end nodes
            const double fa = INTO[ca] * INV[ca], fb = INTO[cb] * INV[cb];
            dn -= fa * TOWARD[ca];
            rh -= fa * RHSN[ca];
            dn -= fb * TOWARD[cb];
            rh -= fb * RHSN[cb];
          }
          if (e < r.w) {
            const int c = CSEC[e] + 1;
            const double f = INTO[c] * INV[c];
            dn -= f * TOWARD[c];
            rh -= f * RHSN[c];
          }
          DN[r.x] = dn;
          RHSN[r.x] = rh;
          INV[r.x] = recip(dn);   // the node's equation is final here
        }
        __syncwarp();
      }
      // (5) substitution, root first: RHSN becomes the node voltage
      if (tid == 0) RHSN[0] = RHSN[0] * INV[0];
      __syncwarp();
      for (int L = 1; L < nlev; ++L) {
        for (int k = LOFF[L] + tid; k < LOFF[L + 1]; k += 32) {
          const int4 r = REC[k];
          RHSN[r.x] = (RHSN[r.x] - TOWARD[r.x] * RHSN[r.y]) * INV[r.x];
        }
        __syncwarp();
      }
    }
    __syncthreads();
    // (6) v = x* + V_start u_start + V_end u_end; capacitive current
    const bool last_step = step == n_steps - 1;
    for (int j = tid; j < nc; j += bs) {
      const int s = __ldg(H.sec_of_comp + c0 + j);
      const double vn = X[j] + RHSN[SPN[s]] * US[j] + RHSN[s + 1] * UE[j];
      if (last_step && write_currents) H.Ic[c0 + j] = H.Cm * (vn - V[j]) / H.dt;
      V[j] = vn;
    }
    // no barrier: a thread owns the same compartments here and in the next step's channel
    // phase (and thread 0 owns compartment 0); the next step's first barrier orders the rest
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
  return 16 * NB + sizeof(double) * (5 * (size_t)nc + 5 * NB + 4 * (size_t)ns) +
         rc_size * 3 * (size_t)nc + sizeof(int32_t) * (4 * (size_t)ns + NB + 1 + (size_t)nlev + 1);
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
  // Neurons whose shared-memory image fits five CTAs per SM run as a second launch of their
  // own size beside the others (on stream2, forked from and joined to the net's stream), so
  // that small neurons do not reserve the largest neuron's shared memory.
  int32_t n_large = 0;                   // CTAs of the first launch (all neurons when 1 class)
  bool large_fits5 = false;              // the first launch's image fits 5 CTAs per SM too
  b2b::HinesDev dev_small{};
  size_t smem_small = 0;
  cudaStream_t stream2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
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
    std::vector<double> low(n_comp, 0.0), diag(n_comp, 0.0), upr(n_comp, 0.0);
    std::vector<int32_t> soc(n_comp), sst(n_sec), sen(n_sec), spn(n_sec);
    std::vector<double> g0(n_sec), gn(n_sec), rfirst(n_sec), rlast(n_sec);
    std::vector<int32_t> child_off, child_sec, level_rec, level_off, lvl_base;
    // r: cross section over half the length; g: axial conductance into c from c - 1
    std::vector<double> area(n_comp), rl(n_comp), g(n_comp + 1, 0.0);
    std::vector<double> soma_area(n_neurons);
    std::vector<int> nlev_of(n_neurons, 0);
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
      // matrix rows (the cable matrix of spatialstateupdate.cu:36-77)
      std::vector<char> first_of_sec(nc, 0);
      for (int s = 0; s < ns; ++s) first_of_sec[sec_start[s0 + s]] = 1;
      for (int64_t c = c0; c < c1; ++c)
        g[c] = first_of_sec[c - c0] ? 0.0 : 1.0 / (Ri * (1.0 / rl[c - 1] + 1.0 / rl[c]));
      g[c1] = 0.0;
      for (int64_t c = c0; c < c1; ++c) {
        low[c] = g[c] / area[c];
        upr[c] = g[c + 1] / area[c];
        diag[c] = -(Cm / dt) - (g[c] + g[c + 1]) / area[c];
      }
      for (int s = 0; s < ns; ++s) {
        const int64_t first = c0 + sec_start[s0 + s];
        const int64_t last = c0 + sec_end[s0 + s] - 1;
        g0[s0 + s] = rl[first] / Ri;
        gn[s0 + s] = rl[last] / Ri;
        diag[first] -= g0[s0 + s] / area[first];
        diag[last] -= gn[s0 + s] / area[last];
        rfirst[s0 + s] = -g0[s0 + s] / area[first];
        rlast[s0 + s] = -gn[s0 + s] / area[last];
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
      nlev_of[b] = nlev;
      const int edge_base = (int)child_sec.size();
      std::vector<int> first_edge(nB + 1);
      for (int i = 0; i < nB; ++i) {
        child_off.push_back((int)child_sec.size());
        first_edge[i] = (int)child_sec.size() - edge_base;
        for (int s : kids[i]) child_sec.push_back(s);
      }
      first_edge[nB] = (int)child_sec.size() - edge_base;
      std::vector<int> order(nB);
      for (int i = 0; i < nB; ++i) order[i] = i;
      std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return depth[a] < depth[c]; });
      lvl_base.push_back((int)level_off.size());
      for (int i : order) {
        level_rec.push_back(i);
        level_rec.push_back(i == 0 ? -1 : spn[s0 + i - 1]);
        level_rec.push_back(first_edge[i]);
        level_rec.push_back(first_edge[i + 1]);
      }
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
    up(&D.low, low); up(&D.diag, diag); up(&D.up, upr); up(&D.sec_of_comp, soc);
    up(&D.sec_start, sst); up(&D.sec_end, sen); up(&D.sec_pnode, spn);
    up(&D.g0, g0); up(&D.gn, gn); up(&D.rhs_first, rfirst); up(&D.rhs_last, rlast);
    up(&D.child_off, child_off); up(&D.child_sec, child_sec);
    up(&D.level_rec, level_rec); up(&D.level_off, level_off);
    // cost of a neuron's step: the node system walks its levels on one warp (~1000 cycles
    // per level, the largest phase), the compartment-parallel phases grow with its size
    std::vector<int32_t> order(n_neurons);
    std::vector<double> cost(n_neurons);
    for (int b = 0; b < n_neurons; ++b) {
      order[b] = b;
      cost[b] = 1000.0 * (lvl_base[b + 1] - lvl_base[b] - 1) +
                15.0 * (double)(comp_off[b + 1] - comp_off[b]);
    }
    // two classes by shared-memory image: those that fit five CTAs per SM, and the rest; each
    // class in decreasing order of cost, the large class first
    int sm_bytes = 0, reserved = 0;
    cudaDeviceGetAttribute(&sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, net->cfg.device);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, net->cfg.device);
    const size_t small_cap = sm_bytes > 0 ? (size_t)(sm_bytes / 5 - reserved) : 0;
    std::vector<char> small(n_neurons, 0);
    int n_small = 0;
    for (int b = 0; b < n_neurons; ++b) {
      const int nc = (int)(comp_off[b + 1] - comp_off[b]), ns = sec_off[b + 1] - sec_off[b];
      small[b] = hines_smem(nc, ns, nlev_of[b], rc) <= small_cap ? 1 : 0;
      n_small += small[b];
    }
    if (n_small == 0 || n_small == n_neurons || smem <= small_cap)
      std::fill(small.begin(), small.end(), 0);   // one class, one launch
    h->large_fits5 = smem <= small_cap;
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t c) {
      if (small[a] != small[c]) return small[a] < small[c];
      return cost[a] > cost[c];
    });
    int n_large = 0, ncs = 0, nss = 0, nls = 0, ncl = 0, nsl = 0, nll = 0;
    for (int b = 0; b < n_neurons; ++b) {
      const int nc = (int)(comp_off[b + 1] - comp_off[b]), ns = sec_off[b + 1] - sec_off[b];
      if (small[b]) {
        ncs = std::max(ncs, nc); nss = std::max(nss, ns); nls = std::max(nls, nlev_of[b]);
      } else {
        ++n_large;
        ncl = std::max(ncl, nc); nsl = std::max(nsl, ns); nll = std::max(nll, nlev_of[b]);
      }
    }
    up(&D.order, order);
    h->n_large = n_large;
    if (n_large < n_neurons) {
      // the large class's image bounds its own arrays; the small class has its own bounds
      D.nc_max = ncl; D.ns_max = nsl; D.nlev_max = nll;
      h->smem = hines_smem(ncl, nsl, nll, rc);
      h->smem_small = hines_smem(ncs, nss, nls, rc);
      if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream2, cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming);
    }
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
    if (n_large < n_neurons) {
      // the small class: the same arrays, its own bounds and its part of the order
      h->dev_small = D;
      h->dev_small.nc_max = ncs; h->dev_small.ns_max = nss; h->dev_small.nlev_max = nls;
      h->dev_small.order = D.order + n_large;
    }
    // shared memory of each kernel variant: the first launch's image for the variant it runs
    // (5 CTAs per SM when its image fits them), the small class's for the other
    const int s5 = (int)std::max(h->large_fits5 ? smem : 0, n_large < n_neurons ? h->smem_small : 0);
    if (e == cudaSuccess && !h->large_fits5)
      e = rc == 4 ? cudaFuncSetAttribute(hines_kernel<float, kHinesLargeCtas>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                  : cudaFuncSetAttribute(hines_kernel<double, kHinesLargeCtas>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess && s5 > 0)
      e = rc == 4 ? cudaFuncSetAttribute(hines_kernel<float, kHinesSmallCtas>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, s5)
                  : cudaFuncSetAttribute(hines_kernel<double, kHinesSmallCtas>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, s5);
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
    cudaStream_t s = h->net->stream;
    const bool two = h->n_large < h->n_neurons;
    if (two) {
      if (cudaEventRecord(h->ev_fork, s) != cudaSuccess) return B2B_ERR_CUDA;
      if (cudaStreamWaitEvent(h->stream2, h->ev_fork, 0) != cudaSuccess) return B2B_ERR_CUDA;
    }
    if (h->channel_dtype == B2B_F32) {
      if (h->n_large > 0 && h->large_fits5)
        hines_kernel<float, kHinesSmallCtas><<<h->n_large, kHinesBlock, h->smem, s>>>(h->dev, k, wc);
      else if (h->n_large > 0)
        hines_kernel<float, kHinesLargeCtas><<<h->n_large, kHinesBlock, h->smem, s>>>(h->dev, k, wc);
      if (two)
        hines_kernel<float, kHinesSmallCtas><<<h->n_neurons - h->n_large, kHinesBlock, h->smem_small,
                              h->stream2>>>(h->dev_small, k, wc);
    } else {
      if (h->n_large > 0 && h->large_fits5)
        hines_kernel<double, kHinesSmallCtas><<<h->n_large, kHinesBlock, h->smem, s>>>(h->dev, k, wc);
      else if (h->n_large > 0)
        hines_kernel<double, kHinesLargeCtas><<<h->n_large, kHinesBlock, h->smem, s>>>(h->dev, k, wc);
      if (two)
        hines_kernel<double, kHinesSmallCtas><<<h->n_neurons - h->n_large, kHinesBlock, h->smem_small,
                               h->stream2>>>(h->dev_small, k, wc);
    }
    if (cudaGetLastError() != cudaSuccess) return B2B_ERR_CUDA;
    if (two) {
      if (cudaEventRecord(h->ev_join, h->stream2) != cudaSuccess) return B2B_ERR_CUDA;
      if (cudaStreamWaitEvent(s, h->ev_join, 0) != cudaSuccess) return B2B_ERR_CUDA;
    }
    h->net->launches += two ? 2 : 1;
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
  if (h->stream2) {
    cudaStreamSynchronize(h->stream2);
    cudaStreamDestroy(h->stream2);
  }
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join) cudaEventDestroy(h->ev_join);
  for (void* a : h->allocs) cudaFree(a);
  delete h;
  return B2B_OK;
}

}  // extern "C"

// ---- the solver's reciprocal against the IEEE quotient ---------------------------------------
namespace b2b {
namespace {
__global__ void recip_selftest_kernel(const double* __restrict__ x, double* __restrict__ y,
                                      int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = recip(x[i]);
}
}  // namespace
}  // namespace b2b

extern "C" b2b_status b2b_recip_selftest(int32_t device, const double* x, double* y,
                                         int64_t n) {
  if (!x || !y || n <= 0) return B2B_ERR_INVALID_ARG;
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess)
    return B2B_ERR_CUDA;
  double *dx = nullptr, *dy = nullptr;
  cudaError_t e = cudaMalloc(&dx, sizeof(double) * n);
  if (e == cudaSuccess) e = cudaMalloc(&dy, sizeof(double) * n);
  if (e == cudaSuccess) e = cudaMemcpy(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    b2b::recip_selftest_kernel<<<256, 256>>>(dx, dy, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(y, dy, sizeof(double) * n, cudaMemcpyDeviceToHost);
  if (dx) cudaFree(dx);
  if (dy) cudaFree(dy);
  cudaSetDevice(prev);
  return e == cudaSuccess ? B2B_OK : B2B_ERR_CUDA;
}
