// Per-neuron update arithmetic shared by the per-step kernels (neuron.cu) and the
// persistent multi-step kernel (fused.cu), so both evaluate exactly the same expressions.
#pragma once
#include "kernels_common.cuh"

namespace b2b {

// Brian2's `timestep(t, dt)` (brian2cuda/cuda_generator.py:997-1006).
__device__ __forceinline__ int64_t timestep_of(double t, double dt) {
  return (int64_t)((t + 1e-3 * dt) / dt);
}

// Exact propagator of dv/dt = (El - v + ke ge + ki gi)/taum, dge/dt = -ge/taue,
// dgi/dt = -gi/taui over one dt (coefficients prepared on the host, LifDev).  Returns the new
// v; advances ge and gi in place.
template <typename R>
__device__ __forceinline__ R lif_advance(const LifDev& g, R v, R& ge, R& gi, bool nr) {
  R vn = dfma((R)g.Bi, gi, dfma((R)g.Be, ge, dfma((R)g.A, v - (R)g.El, (R)g.El)));
  if (g.unless_refractory && !nr) vn = v;
  ge = (R)g.De * ge;
  gi = (R)g.Di * gi;
  return vn;
}

// Exponential Euler: x' = -B/A + (x + B/A) exp(A dt) for dx/dt = A x + B.
template <typename R>
__device__ __forceinline__ R expeuler(R x, R A, R B, R dt) {
  const R BA = B / A;
  return -BA + (BA + x) * dexp(A * dt);
}

// Gating part of the COBAHH update (examples/cobahh.py:159-180): the exponential-Euler step
// of m, h, n over one dt at membrane potential v.  Rates in SI units; the three of the form
// x/(exp(x/a) - 1) go through z/expm1(z) (see z_over_expm1).
template <typename R>
__device__ __forceinline__ void hh_gating(R VT, R v, R& m, R& h, R& n, R dt) {
  // 0.32/mV*(13mV-v+VT)/(exp((13mV-v+VT)/4mV)-1)/ms = 1280 * z/expm1(z), z = (..)/4mV
  const R am = (R)1280 * z_over_expm1(((R)13e-3 - v + VT) / (R)4e-3);
  const R bm = (R)1400 * z_over_expm1((v - VT - (R)40e-3) / (R)5e-3);
  const R ah = (R)128 * dexp(((R)17e-3 - v + VT) / (R)18e-3);
  const R bh = (R)4000 / ((R)1 + dexp(((R)40e-3 - v + VT) / (R)5e-3));
  const R an = (R)160 * z_over_expm1(((R)15e-3 - v + VT) / (R)5e-3);
  const R bn = (R)500 * dexp(((R)10e-3 - v + VT) / (R)40e-3);
  m = expeuler(m, -(am + bm), am, dt);
  h = expeuler(h, -(ah + bh), ah, dt);
  n = expeuler(n, -(an + bn), an, dt);
}

// Membrane part of the COBAHH update: exponential Euler for v with the conductances of the
// gating state at the start of the step.  Returns the new v.
template <typename R>
__device__ __forceinline__ R hh_membrane(const HhDev& g, R v, R m, R h, R n, R ge, R gi, R dt) {
  const R gl = (R)g.gl, Cm = (R)g.Cm;
  const R gna = (R)g.gNa * (m * m * m) * h;
  const R gk = (R)g.gK * (n * n * n * n);
  const R Av = -(gl + ge + gi + gna + gk) / Cm;
  const R Bv = (gl * (R)g.El + ge * (R)g.Ee + gi * (R)g.Ei + gna * (R)g.ENa + gk * (R)g.EK) / Cm;
  return expeuler(v, Av, Bv, dt);
}

// COBAHH over one dt: every right-hand side uses the values at the start of the step.
// Returns the new v; advances m, h, n, ge, gi in place.
template <typename R>
__device__ __forceinline__ R hh_advance(const HhDev& g, R v, R& m, R& h, R& n, R& ge, R& gi,
                                        R dt) {
  const R vn = hh_membrane<R>(g, v, m, h, n, ge, gi, dt);
  hh_gating<R>((R)g.VT, v, m, h, n, dt);
  ge = (R)g.De * ge;
  gi = (R)g.Di * gi;
  return vn;
}

}  // namespace b2b
