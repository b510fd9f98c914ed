// Per-neuron update arithmetic shared by the per-step kernels (neuron.cu) and the one-CTA
// kernel for small networks (small.cu), so both evaluate exactly the same expressions.
#pragma once
#include "kernels_common.cuh"
#include "philox.cuh"

namespace b2b {

// Brian2's not_refractory test, timestep(t - lastspike) >= timestep(refractory) = k, with
// timestep(t, dt) = (int64)((t + 1e-3 dt) / dt) (brian2cuda/cuda_generator.py:997-1006).  The
// division is a product with inv_dt = 1/dt: the quotient is an integer plus 1e-3 (plus the
// rounding of a float32 lastspike, below 1e-3 of a step for t < 100 s), so the one-ulp
// difference between the two forms never changes the truncation.  The elapsed time
// e = t - lastspike is never negative (lastspike starts at -1e4 s and is set to t on a
// spike), so the quotient is positive, its truncation is its floor, and floor(y) >= k exactly
// when y >= k for an integer k: the comparison is made on the quotient, without converting a
// double to a 64-bit integer.
__device__ __forceinline__ bool past_refractory(double e, double dt, double inv_dt,
                                                int64_t k) {
  return (e + 1e-3 * dt) * inv_dt >= (double)k;
}

// Exact propagator of dv/dt = (El + u - v + ke ge + ki gi)/taum, dge/dt = -ge/taue,
// dgi/dt = -gi/taui over one dt (coefficients prepared on the host, LifDev), u held constant
// over the step.  Returns the new v; advances ge and gi in place.
template <typename R>
__device__ __forceinline__ R lif_advance(const LifDev& g, R v, R& ge, R& gi, bool nr,
                                         R u = R(0)) {
  const R El = (R)g.El + u;   // u: TimedArray input (volts), constant over the step
  R vn = dfma((R)g.Bi, gi, dfma((R)g.Be, ge, dfma((R)g.A, v - El, El)));
  if (g.unless_refractory && !nr) vn = v;
  ge = (R)g.De * ge;
  gi = (R)g.Di * gi;
  return vn;
}

// Arithmetic of the COBAHH update.  float64 keeps the correctly rounded library forms.
// float32 uses the hardware units in their flush-to-zero forms (a result below 1.2e-38
// becomes 0; no operand or result of the update comes near that range otherwise): exp(x) as
// 2^(x log2 e) on the ex2 unit (relative error ~1e-6 for the |x| <= 25 the rates reach, from
// the rounding of x log2 e), division as a product with the reciprocal unit's 1/b, and
// division by a literal constant as a product with its rounded reciprocal; all of it is far
// inside the 1e-5 relative tolerance against the float64 oracle.  The flush-to-zero forms
// need no subnormal handling around each ex2 and reciprocal.
__device__ __forceinline__ float ex2_ftz(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_ftz(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float hexp(float x) { return ex2_ftz(x * 1.4426950408889634f); }
__device__ __forceinline__ double hexp(double x) { return exp(x); }
__device__ __forceinline__ float hdiv(float a, float b) { return a * rcp_ftz(b); }
__device__ __forceinline__ double hdiv(double a, double b) { return a / b; }
// x / c for a literal c.
__device__ __forceinline__ float hdivc(float x, double c) { return x * (float)(1.0 / c); }
__device__ __forceinline__ double hdivc(double x, double c) { return x / c; }
// z / (exp(z) - 1) with its z = 0 limit.  float32: near 0 the Taylor series of the
// generating function of the Bernoulli numbers, sum_k B_k z^k / k!
// (1 - z/2 + z^2/12 - z^4/720 + z^6/30240 - z^8/1209600, truncation < 1e-10 for |z| < 1/2);
// elsewhere exp(z) - 1 >= 0.39 in magnitude, so ex2's error is not amplified by more than 2.5.
__device__ __forceinline__ float hz_over_expm1(float z) {
  if (fabsf(z) < 0.5f) {
    const float z2 = z * z;
    const float even = fmaf(z2, fmaf(z2, fmaf(z2, fmaf(z2, -1.f / 1209600.f, 1.f / 30240.f),
                                               -1.f / 720.f), 1.f / 12.f), 1.f);
    return fmaf(z, -0.5f, even);
  }
  return z * rcp_ftz(hexp(z) - 1.f);
}
__device__ __forceinline__ double hz_over_expm1(double z) { return z_over_expm1(z); }

// Exponential Euler: x' = -B/A + (x + B/A) exp(A dt) for dx/dt = A x + B.
template <typename R>
__device__ __forceinline__ R expeuler(R x, R A, R B, R dt) {
  const R BA = hdiv(B, A);
  return -BA + (BA + x) * hexp(A * dt);
}

// Gating part of the COBAHH update (examples/cobahh.py:159-180): the exponential-Euler step
// of m, h, n over one dt at membrane potential v.  Rates in SI units; the three of the form
// x/(exp(x/a) - 1) go through z/(exp(z) - 1) (hz_over_expm1, Brian2's exprel).
template <typename R>
__device__ __forceinline__ void hh_gating(R VT, R v, R& m, R& h, R& n, R dt) {
  // 0.32/mV*(13mV-v+VT)/(exp((13mV-v+VT)/4mV)-1)/ms = 1280 * z/expm1(z), z = (..)/4mV
  const R am = (R)1280 * hz_over_expm1(hdivc((R)13e-3 - v + VT, 4e-3));
  const R bm = (R)1400 * hz_over_expm1(hdivc(v - VT - (R)40e-3, 5e-3));
  const R ah = (R)128 * hexp(hdivc((R)17e-3 - v + VT, 18e-3));
  const R bh = hdiv((R)4000, (R)1 + hexp(hdivc((R)40e-3 - v + VT, 5e-3)));
  const R an = (R)160 * hz_over_expm1(hdivc((R)15e-3 - v + VT, 5e-3));
  const R bn = (R)500 * hexp(hdivc((R)10e-3 - v + VT, 40e-3));
  m = expeuler(m, -(am + bm), am, dt);
  h = expeuler(h, -(ah + bh), ah, dt);
  n = expeuler(n, -(an + bn), an, dt);
}

// A group's HH constants in the arithmetic type R of the update (float32: the host-rounded
// copies, float64: the originals) with its refractory period and range.
template <typename R>
struct HhRun {
  R Cm, gl, El, EK, ENa, gNa, gK, VT, Ee, Ei, De, Di, Vthr, inv_Cm;
  int64_t ref_steps, offset, n;
};
__device__ __forceinline__ HhRun<float> hh_run(const HhDev& g, float) {
  const HhFloat& f = g.f;
  return {f.Cm, f.gl, f.El, f.EK, f.ENa, f.gNa, f.gK, f.VT, f.Ee, f.Ei, f.De, f.Di, f.Vthr,
          f.inv_Cm, g.ref_steps, g.offset, g.n};
}
__device__ __forceinline__ HhRun<double> hh_run(const HhDev& g, double) {
  return {g.Cm, g.gl, g.El, g.EK, g.ENa, g.gNa, g.gK, g.VT, g.Ee, g.Ei, g.De, g.Di, g.Vthr,
          g.inv_Cm, g.ref_steps, g.offset, g.n};
}

// TimedArray input of a group at step ts for its neuron `local` (the role of the function
// brian2cuda/timedarray.py:10-58 generates: the array's time step holding t, clamped to the
// last row; one column for the whole group, or one per neuron).  The row is computed from
// the integer step, since the time grids are aligned (b2b_timedarray checks it).  Padding
// neurons past the group's end read its last column; their results are never used.
template <typename R>
__device__ __forceinline__ R timed_input(const TimedInput& ta, int64_t ts, int64_t local) {
  if (!ta.val) return (R)0;
  int64_t row = ts * ta.mul / ta.div;
  if (row >= ta.rows) row = ta.rows - 1;
  const int64_t col = ta.cols == 1 ? 0 : (local < ta.cols ? local : ta.cols - 1);
  return __ldg(static_cast<const R*>(ta.val) + row * ta.cols + col);
}

// 1/Cm (float32, from the group's precomputed reciprocal) or division by Cm (float64).
__device__ __forceinline__ float per_cm(float x, const HhRun<float>& g) { return x * g.inv_Cm; }
__device__ __forceinline__ double per_cm(double x, const HhRun<double>& g) { return x / g.Cm; }

// Membrane part of the COBAHH update: exponential Euler for v with the conductances of the
// gating state at the start of the step.  Returns the new v.
// One Binomial(n, p) draw of a PoissonInput for the group-local neuron `local` at step ts
// (the role of the inversion sampler brian2cuda/binomial.py:55-90 generates for
// BinomialFunction, restated as sequential-search inversion, Devroye, "Non-Uniform Random
// Variate Generation", 1986, ch. X.4): u uniform in (0, 1) from one Philox-4x32-10 word;
// subtract P(X = 0), P(X = 1), ... from u until it is no longer above the next probability,
// with P(X = x) = P(X = x - 1) (a / x - s).  Every operation is an IEEE double operation
// (no fused multiply-add can form), and q^n, s and a come from the host, so the CPU
// oracle's restatement draws the same X.  At most n steps; mass lost to rounding goes to n.
static __device__ __noinline__ int64_t poisson_input_draw(const PoissonIn& p, int64_t ts,
                                                      int64_t local) {
  const U32x4 w = philox4x32_10(U32x4{(uint32_t)local, (uint32_t)ts,
                                      (uint32_t)((uint64_t)ts >> 32), p.id}, p.k0, p.k1);
  double u = ((double)w.x + 0.5) * 0x1p-32;
  double r = p.qn;
  int64_t x = 0;
  while (u > r && x < p.n) {
    u = __dsub_rn(u, r);
    ++x;
    r = __dmul_rn(r, __dsub_rn(__ddiv_rn(p.a, (double)x), p.s));
  }
  return p.reverse ? p.n - x : x;
}

__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

// The group's PoissonInputs for one neuron: variable += weight * X, in the group's dtype, the
// product rounded before the sum (as the oracle computes it; no fused multiply-add).
template <typename R>
__device__ __forceinline__ void add_poisson_inputs(const PoissonInputs& pin, int64_t ts,
                                                   int64_t local, R& v, R& ge, R& gi) {
  for (int k = 0; k < pin.count; ++k) {
    const PoissonIn& p = pin.in[k];
    const R add = mul_rn((R)poisson_input_draw(p, ts, local), (R)p.weight);
    if (p.var == B2B_VAR_V) v += add;
    else if (p.var == B2B_VAR_GE) ge += add;
    else gi += add;
  }
}

// I: external current (amperes) over the step, from a TimedArray.
template <typename R>
__device__ __forceinline__ R hh_membrane(const HhRun<R>& g, R v, R m, R h, R n, R ge, R gi,
                                         R dt, R I = R(0)) {
  const R gl = (R)g.gl;
  const R gna = (R)g.gNa * (m * m * m) * h;
  const R gk = (R)g.gK * (n * n * n * n);
  const R Av = -per_cm(gl + ge + gi + gna + gk, g);
  const R Bv = per_cm(gl * (R)g.El + ge * (R)g.Ee + gi * (R)g.Ei + gna * (R)g.ENa + gk * (R)g.EK + I, g);
  return expeuler(v, Av, Bv, dt);
}

// COBAHH over one dt: every right-hand side uses the values at the start of the step.
// Returns the new v; advances m, h, n, ge, gi in place.
template <typename R>
__device__ __forceinline__ R hh_advance(const HhRun<R>& g, R v, R& m, R& h, R& n, R& ge, R& gi,
                                        R dt, R I = R(0)) {
  const R vn = hh_membrane<R>(g, v, m, h, n, ge, gi, dt, I);
  hh_gating<R>((R)g.VT, v, m, h, n, dt);
  ge = (R)g.De * ge;
  gi = (R)g.Di * gi;
  return vn;
}

}  // namespace b2b
