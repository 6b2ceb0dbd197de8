// Distance arithmetic of the reference's evalPoint (kernel.cu:307-365),
// restated exactly: every rounding step is an explicit intrinsic.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "gsj_common.cuh"
#include "gsj_fp.cuh"

namespace gsj {

// Contraction policy of the reference's device arithmetic.  The source
// accumulates `acc += d*d` from acc = 0; nvcc turns it into fused
// multiply-adds in a precision-dependent way, pinned against the reference's
// own builds (tests/golden/ref_pins.json):
//   kPolF32  0 + d*d stays fma(d, d, 0), so every later term is fused into
//            the running value (float).
//   kPolF64  0 + d*d folds to a pending product.  When both operands of an
//            addition are pending products, the accumulator's product is
//            fused in `acc += d*d` (runningTotalDist / runningDist[j]
//            chains), and the added register's product is fused in the
//            cross-register sums `runningDist[0] += runningDist[j]` (double).
enum Policy : int { kPolF32 = 0, kPolF64 = 1 };

template <typename T, int POL>
struct Acc {
    static constexpr bool FOLD0 = POL == kPolF64;
    static constexpr bool CHAIN_LEFT = true;   // acc += d*d with acc pending: fuse acc's product
    static constexpr bool CROSS_LEFT = false;  // acc += other acc, both pending: fuse the other's
    T v, d;
    int st;  // 0: literal zero, 1: pending product d*d (value v), 2: value v
    __device__ __forceinline__ Acc() : v(T(0)), d(T(0)), st(0) {}
    __device__ __forceinline__ void add_prod(T dd) {
        if (st == 0) {
            if (FOLD0) {
                st = 1;
                d = dd;
                v = FP<T>::mul(dd, dd);
            } else {
                st = 2;
                v = FP<T>::fma(dd, dd, T(0));
            }
        } else if (FOLD0 && st == 1) {
            st = 2;
            v = CHAIN_LEFT ? FP<T>::fma(d, d, FP<T>::mul(dd, dd)) : FP<T>::fma(dd, dd, v);
        } else {
            v = FP<T>::fma(dd, dd, v);
        }
    }
    __device__ __forceinline__ void add_acc(const Acc& o) {
        if (o.st == 0) return;
        if (st == 0) {
            *this = o;
            return;
        }
        if (FOLD0 && st == 1 && o.st == 1) {
            v = CROSS_LEFT ? FP<T>::fma(d, d, o.v) : FP<T>::fma(o.d, o.d, v);
        } else if (FOLD0 && o.st == 1) {
            v = FP<T>::fma(o.d, o.d, v);
        } else if (FOLD0 && st == 1) {
            v = FP<T>::fma(d, d, o.v);
        } else {
            v = FP<T>::add(v, o.v);
        }
        st = 2;
    }
};

// Squared distance in the reference's order with the candidate row in
// registers (NT = n known at compile time; sequential model only).
template <typename T, int NT, int POL>
__device__ __forceinline__ T sqdist_seq_reg(const T* __restrict__ q, const T (&c)[NT]) {
    Acc<T, POL> s;
#pragma unroll
    for (int l = 0; l < NT; l++) s.add_prod(FP<T>::sub(c[l], q[l]));
    return s.v;
}

// Generic n: candidate row and query row in shared memory.  `valid` is the
// lane's vote input for the warp-wide early exit; an exit never changes a
// decision because every model's running sum only grows once it is above thr.
template <typename T, int MODEL, int POL>
__device__ __forceinline__ T sqdist_generic(const T* __restrict__ q, const T* __restrict__ c, uint32_t n,
                                            uint32_t ilp, T thr, bool valid) {
    const unsigned FULL = 0xffffffffu;
    if (MODEL == kSeq) {
        // kernel.cu:346-356
        Acc<T, POL> s;
        for (uint32_t l = 0; l < n; l++) {
            s.add_prod(FP<T>::sub(c[l], q[l]));
            if ((l & 7u) == 7u && __all_sync(FULL, !valid || s.v > thr)) break;
        }
        return s.v;
    } else if (MODEL == kIlp) {
        // runningDist[j] accumulates dims l == j (mod ILP); then summed in j order (kernel.cu:312-341)
        Acc<T, POL> s;
        for (uint32_t j = 0; j < ilp; j++) {
            Acc<T, POL> r;
            for (uint32_t l = j; l < n; l += ilp) r.add_prod(FP<T>::sub(c[l], q[l]));
            if (j == 0) s = r;
            else s.add_acc(r);
        }
        return s.v;
    } else {
        // SHORTCIRCUIT with ILP (kernel.cu:320-334): per block, runningDist[0]
        // takes the block's first square, then the other registers are added.
        Acc<T, POL> r0;
        for (uint32_t l = 0; l < n; l += ilp) {
            r0.add_prod(FP<T>::sub(c[l], q[l]));
            for (uint32_t j = 1; j < ilp && l + j < n; j++) {
                Acc<T, POL> rj;
                rj.add_prod(FP<T>::sub(c[l + j], q[l + j]));
                r0.add_acc(rj);
            }
            if (__all_sync(FULL, !valid || r0.v > thr)) break;
        }
        return r0.v;
    }
}

}  // namespace gsj

namespace gsj {

// The same models for one thread on its own (no warp-wide early exit, so it
// may run in divergent code): q and c are rows of n values in global memory.
// Leaving out the early exit never changes a decision.
template <typename T, int MODEL, int POL>
__device__ __forceinline__ T sqdist_lane(const T* __restrict__ q, const T* __restrict__ c, uint32_t n,
                                         uint32_t ilp) {
    if (MODEL == kSeq) {
        Acc<T, POL> s;
        for (uint32_t l = 0; l < n; l++) s.add_prod(FP<T>::sub(c[l], q[l]));
        return s.v;
    } else if (MODEL == kIlp) {
        Acc<T, POL> s;
        for (uint32_t j = 0; j < ilp; j++) {
            Acc<T, POL> r;
            for (uint32_t l = j; l < n; l += ilp) r.add_prod(FP<T>::sub(c[l], q[l]));
            if (j == 0) s = r;
            else s.add_acc(r);
        }
        return s.v;
    } else {
        Acc<T, POL> r0;
        for (uint32_t l = 0; l < n; l += ilp) {
            r0.add_prod(FP<T>::sub(c[l], q[l]));
            for (uint32_t j = 1; j < ilp && l + j < n; j++) {
                Acc<T, POL> rj;
                rj.add_prod(FP<T>::sub(c[l + j], q[l + j]));
                r0.add_acc(rj);
            }
        }
        return r0.v;
    }
}

}  // namespace gsj
