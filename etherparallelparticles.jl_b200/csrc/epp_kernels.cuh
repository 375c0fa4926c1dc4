// epp_kernels.cuh -- the SPH smoothing kernels of src/SPH/Kernel/*.jl.
//
// For each kernel: the value W(r, hinv) (`_value`), the gradient dW/dr (`_gradient`), dW/dr
// divided by r in closed form (what the pair terms use: no division by r per pair), and W at
// r = 0 (`_value0`, Kernel.jl:16-22: sigma * hinv^N for every kernel).  q = r * hinv; the support
// radius is 2 h except for the Gaussian (3 h, truncated in practice by the 2 h search criterion).
// Normalisation sigma_N and the polynomial constants are those of the reference files.
#pragma once
#include "epp_math.cuh"

namespace epp {

// sigma_N: WendlandC2.jl:12-14, CubicSpline.jl:12-14, Gaussian.jl:12-14, WendlandC4.jl:12-14
template <int D>
__device__ __forceinline__ float kern_sigma(int kind) {
    constexpr double pi = 3.14159265358979323846;
    switch (kind) {
        case EPP_KERNEL_CUBIC_SPLINE: return D == 2 ? (float)(10.0 / 7.0 / pi) : (float)(1.0 / pi);
        case EPP_KERNEL_GAUSSIAN: return D == 2 ? (float)(1.0 / pi) : (float)(1.0 / (pi * 1.7724538509055160273));
        case EPP_KERNEL_WENDLAND_C4: return D == 2 ? (float)(9.0 / 4.0 / pi) : (float)(495.0 / 256.0 / pi);
        default: return D == 2 ? (float)(7.0 / 4.0 / pi) : (float)(21.0 / 16.0 / pi);
    }
}

// W(r, hinv)
template <int D>
__device__ __forceinline__ float kern_value(int kind, float r, float hinv) {
    const float q = r * hinv;
    const float s = kern_sigma<D>(kind) * powi(hinv, D);
    switch (kind) {
        case EPP_KERNEL_CUBIC_SPLINE:   // CubicSpline.jl:16-30
            if (q < 1.0f) return s * (3.0f * q * q * (q - 2.0f) + 4.0f) * 0.25f;
            if (q < 2.0f) return s * powi(2.0f - q, 3) * 0.25f;
            return 0.0f;
        case EPP_KERNEL_GAUSSIAN:   // Gaussian.jl:16-26
            return q < 3.0f ? s * expf(-q * q) : 0.0f;
        case EPP_KERNEL_WENDLAND_C4:   // WendlandC4.jl:16-30
            return q < 2.0f ? s * powi(2.0f - q, 6) * (q * (35.0f * q + 36.0f) + 12.0f) * 0.0013020833333333333f
                            : 0.0f;
        default:   // WendlandC2.jl:16-26
            return q < 2.0f ? s * powi(2.0f - q, 4) * (1.0f + 2.0f * q) * 0.0625f : 0.0f;
    }
}

// dW/dr
template <int D>
__device__ __forceinline__ float kern_gradient(int kind, float r, float hinv) {
    const float q = r * hinv;
    const float s = kern_sigma<D>(kind) * powi(hinv, D + 1);
    switch (kind) {
        case EPP_KERNEL_CUBIC_SPLINE:   // CubicSpline.jl:40-54
            if (q < 1.0f) return s * q * (3.0f * q - 4.0f) * 0.75f;
            if (q < 2.0f) return -s * (2.0f - q) * (2.0f - q) * 0.75f;
            return 0.0f;
        case EPP_KERNEL_GAUSSIAN:   // Gaussian.jl:36-46
            return q < 3.0f ? -2.0f * s * q * expf(-q * q) : 0.0f;
        case EPP_KERNEL_WENDLAND_C4:   // WendlandC4.jl:40-56
            return q < 2.0f ? -s * q * (0.3645833333333333f * q + 0.14583333333333334f) * powi(2.0f - q, 5) : 0.0f;
        default:   // WendlandC2.jl:36-46
            return q < 2.0f ? -s * 0.625f * q * powi(2.0f - q, 3) : 0.0f;
    }
}

// (dW/dr) / r from q and hinv (q / r = hinv), 0 outside the support
template <int D>
__device__ __forceinline__ float kern_dwr(int kind, float q, float hinv) {
    const float s = kern_sigma<D>(kind) * powi(hinv, D + 2);
    switch (kind) {
        case EPP_KERNEL_CUBIC_SPLINE:
            if (q < 1.0f) return s * (3.0f * q - 4.0f) * 0.75f;
            if (q < 2.0f) return __fdividef(-s * (2.0f - q) * (2.0f - q) * 0.75f, q);   // a scale, no cancellation
            return 0.0f;
        case EPP_KERNEL_GAUSSIAN:
            return q < 3.0f ? -2.0f * s * expf(-q * q) : 0.0f;
        case EPP_KERNEL_WENDLAND_C4:
            return q < 2.0f ? -s * (0.3645833333333333f * q + 0.14583333333333334f) * powi(2.0f - q, 5) : 0.0f;
        default:
            return q < 2.0f ? -s * 0.625f * powi(2.0f - q, 3) : 0.0f;
    }
}

// W(0, hinv) = sigma * hinv^N (Kernel.jl:16-22)
template <int D>
__device__ __forceinline__ float kern_value0(int kind, float hinv) {
    return kern_sigma<D>(kind) * powi(hinv, D);
}

}  // namespace epp
