"""Writes caps_b200/csrc/ewald_fit.cuh: rational fits for the FP32 pair kernel's Ewald / damped-shifted real-space terms.

With u = (kappa r)^2 the real-space pair terms are
    E = qq (1/r - kappa g(u)),            g(u) = erf(sqrt u) / sqrt u
    F = qq (1/r^3 - kappa^3 h(u)),        h(u) = (g(u) - (2/sqrt(pi)) exp(-u)) / u        (F = -(dE/dr)/r)
Both are smooth in u. Each is fitted on u in [0, 16] (kappa r_c <= 4, i.e. erfc(kappa r_c) >= 1.5e-8) as P(t)/Q(t),
t = u/16, Q(0) = 1, by Sanathanan-Koerner iteration with Lawson reweighting towards minimax relative error. The kernel
evaluates them with FMAs and one division, instead of erfc and exp per pair; beyond kappa r_c = 4 the engine keeps the
library erfcf form.

    python caps_b200/fits/make_ewald_fit.py
"""
from __future__ import annotations

from math import factorial
from pathlib import Path

import numpy as np
from scipy.special import erf

U = 16.0
OUT = Path(__file__).resolve().parent.parent / "csrc" / "ewald_fit.cuh"


def g(u):
    z = np.sqrt(u)
    return np.where(u < 1e-14, 2 / np.sqrt(np.pi), erf(z) / np.where(z > 0, z, 1))


def h(u):
    z = np.sqrt(np.maximum(u, 1e-300))
    with np.errstate(all="ignore"):
        v = (erf(z) / z - 2 / np.sqrt(np.pi) * np.exp(-u)) / u
    s = sum((-1) ** (n + 1) * 2 * n * u ** (n - 1) / (factorial(n) * (2 * n + 1)) for n in range(1, 16)) * 2 / np.sqrt(np.pi)
    return np.where(u < 2e-2, s, v)


def fit(f, m: int, k: int, iters: int = 60):
    t = np.linspace(0, 1, 6001)
    y = f(t * U)
    w = np.ones_like(t)
    q = np.ones_like(t)
    for _ in range(iters):
        A = np.hstack([t[:, None] ** np.arange(m + 1), -(y[:, None]) * t[:, None] ** np.arange(1, k + 1)])
        W = (w / q)[:, None]
        sol, *_ = np.linalg.lstsq(A * W, y * (w / q), rcond=None)
        p, qq = sol[:m + 1], np.concatenate([[1.0], sol[m + 1:]])
        q = np.polyval(qq[::-1], t)
        err = (np.polyval(p[::-1], t) / q - y) / y
        w = w * (1 + 3 * np.abs(err) / np.abs(err).max())
    assert q.min() > 0.5, "denominator must stay positive"
    return p, qq, float(np.abs(err).max())


def f32_error(f, p, q) -> float:
    t = np.linspace(0, 1, 200001).astype(np.float32)
    pv = np.zeros_like(t)
    for c in p[::-1]:
        pv = pv * t + np.float32(c)
    qv = np.zeros_like(t)
    for c in q[::-1]:
        qv = qv * t + np.float32(c)
    y = f(t.astype(np.float64) * U)
    return float(np.max(np.abs((pv / qv).astype(np.float64) - y) / np.abs(y)))


def main():
    hp, hq, he = fit(h, 7, 5)
    gp, gq, ge = fit(g, 6, 5)
    def horner(v) -> str:   # explicit nested FMAs: the coefficients become instruction immediates
        e = f"{float(v[-1]):.9e}f"
        for c in v[-2::-1]:
            e = f"fmaf({e}, t, {float(c):.9e}f)"
        return e

    def horner2(v) -> str:   # the same on both lanes of an f32x2 pair (sm_100 packed FP32 arithmetic)
        e = f"make_float2({float(v[-1]):.9e}f, {float(v[-1]):.9e}f)"
        for c in v[-2::-1]:
            e = f"__ffma2_rn({e}, t, make_float2({float(c):.9e}f, {float(c):.9e}f))"
        return e

    text = f"""// Generated by caps_b200/fits/make_ewald_fit.py: rational fits on u = (kappa r)^2 in [0, {U:g}], t = u / {U:g}.
//   g(u) = erf(sqrt u) / sqrt u                       fit max relative error {ge:.1e}, float evaluation {f32_error(g, gp, gq):.1e}
//   h(u) = (g(u) - 2 exp(-u) / sqrt(pi)) / u          fit max relative error {he:.1e}, float evaluation {f32_error(h, hp, hq):.1e}
#pragma once
namespace capsb {{
constexpr float kEwUMax = {U:.1f}f;
__device__ __forceinline__ float ew_h(float t) {{ return __fdividef({horner(hp)}, {horner(hq)}); }}
__device__ __forceinline__ float ew_g(float t) {{ return __fdividef({horner(gp)}, {horner(gq)}); }}
// the SFU's approximate reciprocal with denormals flushed (the denominators lie in [1, 300])
__device__ __forceinline__ float rcp_ftz(float x) {{
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}}
// both fits on a pair of arguments at once (packed FP32 multiply-adds; the two reciprocals are taken separately)
__device__ __forceinline__ float2 ew_h2(float2 t) {{
  const float2 n = {horner2(hp)};
  const float2 d = {horner2(hq)};
  return __fmul2_rn(n, make_float2(rcp_ftz(d.x), rcp_ftz(d.y)));
}}
__device__ __forceinline__ float2 ew_g2(float2 t) {{
  const float2 n = {horner2(gp)};
  const float2 d = {horner2(gq)};
  return __fmul2_rn(n, make_float2(rcp_ftz(d.x), rcp_ftz(d.y)));
}}
}}  // namespace capsb
"""
    OUT.write_text(text)
    print(f"wrote {OUT}: h {he:.1e} (f32 {f32_error(h, hp, hq):.1e}), g {ge:.1e} (f32 {f32_error(g, gp, gq):.1e})")


if __name__ == "__main__":
    main()
