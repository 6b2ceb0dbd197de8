// Explicitly rounded arithmetic.  Every operation of the restated reference
// arithmetic is spelled out with a round-to-nearest intrinsic so the compiler
// can neither contract nor reassociate it: the reference's device code fuses
// `s += d*d` into one fma (written here as FP<T>::fma), and its host code
// (index build, REORDER statistic) does not fuse at all.
#pragma once
#include <cuda_runtime.h>

namespace gsj {

template <typename T>
struct FP;

template <>
struct FP<float> {
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
    static __device__ __forceinline__ unsigned to_uint_rz(float a) { return __float2uint_rz(a); }
};

template <>
struct FP<double> {
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
    static __device__ __forceinline__ unsigned to_uint_rz(double a) { return __double2uint_rz(a); }
};

}  // namespace gsj
