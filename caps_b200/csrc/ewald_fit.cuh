// Generated by caps_b200/fits/make_ewald_fit.py: rational fits on u = (kappa r)^2 in [0, 16], t = u / 16.
//   g(u) = erf(sqrt u) / sqrt u                       fit max relative error 2.0e-09, float evaluation 3.5e-07
//   h(u) = (g(u) - 2 exp(-u) / sqrt(pi)) / u          fit max relative error 1.1e-08, float evaluation 3.9e-07
#pragma once
namespace capsb {
constexpr float kEwUMax = 16.0f;
__device__ __forceinline__ float ew_h(float t) { return __fdividef(fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(-1.545778376e-01f, t, 1.023093715e+00f), t, -3.035759399e+00f), t, 5.564720173e+00f), t, -4.039556622e+00f), t, 5.280225867e+00f), t, -1.072285143e+00f), t, 7.522527865e-01f), fmaf(fmaf(fmaf(fmaf(fmaf(7.518246663e+01f, t, 9.347137021e+01f), t, 6.789361603e+01f), t, 3.063738701e+01f), t, 8.174574414e+00f), t, 1.000000000e+00f)); }
__device__ __forceinline__ float ew_g(float t) { return __fdividef(fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(-2.214897670e-01f, t, 4.912257566e+00f), t, 2.487786276e+01f), t, 1.576802594e+01f), t, 1.390512202e+01f), t, 2.963256597e+00f), t, 1.128379169e+00f), fmaf(fmaf(fmaf(fmaf(fmaf(6.617541336e+01f, t, 8.569271198e+01f), t, 6.333271079e+01f), t, 2.917337202e+01f), t, 7.959452403e+00f), t, 1.000000000e+00f)); }
// the SFU's approximate reciprocal with denormals flushed (the denominators lie in [1, 300])
__device__ __forceinline__ float rcp_ftz(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
// both fits on a pair of arguments at once (packed FP32 multiply-adds; the two reciprocals are taken separately)
__device__ __forceinline__ float2 ew_h2(float2 t) {
  const float2 n = __ffma2_rn(__ffma2_rn(__ffma2_rn(__ffma2_rn(__ffma2_rn(__ffma2_rn(__ffma2_rn(make_float2(-1.545778376e-01f, -1.545778376e-01f), t, make_float2(1.023093715e+00f, 1.023093715e+00f)), t, make_float2(-3.035759399e+00f, -3.035759399e+00f)), t, make_float2(5.564720173e+00f, 5.564720173e+00f)), t, make_float2(-4.039556622e+00f, -4.039556622e+00f)), t, make_float2(5.280225867e+00f, 5.280225867e+00f)), t, make_float2(-1.072285143e+00f, -1.072285143e+00f)), t, make_float2(7.522527865e-01f, 7.522527865e-01f));
  const float2 d = __ffma2_rn(__ffma2_rn(__ffma2_rn(__ffma2_rn(__ffma2_rn(make_float2(7.518246663e+01f, 7.518246663e+01f), t, make_float2(9.347137021e+01f, 9.347137021e+01f)), t, make_float2(6.789361603e+01f, 6.789361603e+01f)), t, make_float2(3.063738701e+01f, 3.063738701e+01f)), t, make_float2(8.174574414e+00f, 8.174574414e+00f)), t, make_float2(1.000000000e+00f, 1.000000000e+00f));
  return __fmul2_rn(n, make_float2(rcp_ftz(d.x), rcp_ftz(d.y)));
}
__device__ __forceinline__ float2 ew_g2(float2 t) {
  const float2 n = __ffma2_rn(__ffma2_rn(__ffma2_rn(__ffma2_rn(__ffma2_rn(__ffma2_rn(make_float2(-2.214897670e-01f, -2.214897670e-01f), t, make_float2(4.912257566e+00f, 4.912257566e+00f)), t, make_float2(2.487786276e+01f, 2.487786276e+01f)), t, make_float2(1.576802594e+01f, 1.576802594e+01f)), t, make_float2(1.390512202e+01f, 1.390512202e+01f)), t, make_float2(2.963256597e+00f, 2.963256597e+00f)), t, make_float2(1.128379169e+00f, 1.128379169e+00f));
  const float2 d = __ffma2_rn(__ffma2_rn(__ffma2_rn(__ffma2_rn(__ffma2_rn(make_float2(6.617541336e+01f, 6.617541336e+01f), t, make_float2(8.569271198e+01f, 8.569271198e+01f)), t, make_float2(6.333271079e+01f, 6.333271079e+01f)), t, make_float2(2.917337202e+01f, 2.917337202e+01f)), t, make_float2(7.959452403e+00f, 7.959452403e+00f)), t, make_float2(1.000000000e+00f, 1.000000000e+00f));
  return __fmul2_rn(n, make_float2(rcp_ftz(d.x), rcp_ftz(d.y)));
}
}  // namespace capsb
