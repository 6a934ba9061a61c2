// Types of the device PME shared by the host engine and the PME kernels (pme.cuh).
#pragma once
#include "common.cuh"

namespace capsb {

constexpr int kMaxRadices = 16;
constexpr int kMaxOrder = 8;

template <class R> struct Cpx;
template <> struct Cpx<float> { using T = float2; };
template <> struct Cpx<double> { using T = double2; };

template <class T> __device__ __forceinline__ T cmul(T a, T b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
template <class T> __device__ __forceinline__ T cadd(T a, T b) { return {a.x + b.x, a.y + b.y}; }
template <class T> __device__ __forceinline__ T csub(T a, T b) { return {a.x - b.x, a.y - b.y}; }

template <class R>
struct FftPlan {
  int n, nst;
  int rad[kMaxRadices];
  const typename Cpx<R>::T* tw;   // exp(sign 2 pi i k / n), k < n
  int sign;                        // +1 / -1 (the sign of tw)
};

}  // namespace capsb
