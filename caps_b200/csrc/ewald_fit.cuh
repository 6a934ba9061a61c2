// Generated by caps_b200/fits/make_ewald_fit.py: rational fits on u = (kappa r)^2 in [0, 16], t = u / 16.
//   g(u) = erf(sqrt u) / sqrt u                       fit max relative error 2.0e-09, float evaluation 3.5e-07
//   h(u) = (g(u) - 2 exp(-u) / sqrt(pi)) / u          fit max relative error 1.1e-08, float evaluation 3.9e-07
#pragma once
namespace capsb {
constexpr float kEwUMax = 16.0f;
__device__ __forceinline__ float ew_h(float t) { return __fdividef(fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(-1.545778376e-01f, t, 1.023093715e+00f), t, -3.035759399e+00f), t, 5.564720173e+00f), t, -4.039556622e+00f), t, 5.280225867e+00f), t, -1.072285143e+00f), t, 7.522527865e-01f), fmaf(fmaf(fmaf(fmaf(fmaf(7.518246663e+01f, t, 9.347137021e+01f), t, 6.789361603e+01f), t, 3.063738701e+01f), t, 8.174574414e+00f), t, 1.000000000e+00f)); }
__device__ __forceinline__ float ew_g(float t) { return __fdividef(fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(-2.214897670e-01f, t, 4.912257566e+00f), t, 2.487786276e+01f), t, 1.576802594e+01f), t, 1.390512202e+01f), t, 2.963256597e+00f), t, 1.128379169e+00f), fmaf(fmaf(fmaf(fmaf(fmaf(6.617541336e+01f, t, 8.569271198e+01f), t, 6.333271079e+01f), t, 2.917337202e+01f), t, 7.959452403e+00f), t, 1.000000000e+00f)); }
}  // namespace capsb
