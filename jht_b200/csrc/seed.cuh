// Recursion seeds shared by the Legendre kernels (legendre.cu) and the tensor-core
// adjoint's block-state kernel (tc_adjoint.cu): the log of the first value of each
// column, as jht's NumPy plan rounds it, turned into the scaled representation.
#pragma once

#include <cuda_runtime.h>

#include "jhtb_internal.cuh"

namespace jhtb {

// sign * exp(lg) as mant * 2^(800 sc) with |mant| in [2^-400, 2^400), sc <= 0.
// The reduction lg - sc * 800 ln2 uses a two-part constant so it adds no error.
__device__ __forceinline__ void make_seed(double lg, double sign, double &mant, int &sc) {
    if (!(lg > -1.0e300)) {  // log(0): exact zero at a pole
        mant = 0.0;
        sc = 0;
        return;
    }
    int k = (int)floor((lg + kLn2x400) / (kLogScaleHi + kLogScaleLo));
    if (k > 0) k = 0;
    const double dk = (double)k;
    const double r = __dadd_rn(__dadd_rn(lg, -__dmul_rn(dk, kLogScaleHi)), -__dmul_rn(dk, kLogScaleLo));
    mant = sign * exp(r);
    sc = k;
}

// log|seed| for ring t: spin 0 (_recursion.py:315-317), spin +-2 (:181-187).
// Unfused mul/add so the value is rounded exactly as jht's NumPy plan rounds it.
__device__ __forceinline__ double seed_log0(const SeedParam &sp, int m, double logsin) {
    return m == 0 ? sp.lf[0] : __dadd_rn(sp.lf[0], __dmul_rn((double)m, logsin));
}
__device__ __forceinline__ double seed_log2(const SeedParam &sp, int h, double lch, double lsh) {
    double v = sp.lf[h];
    if (sp.pc[h] > 0) v = __dadd_rn(v, __dmul_rn((double)sp.pc[h], lch));
    if (sp.ps[h] > 0) v = __dadd_rn(v, __dmul_rn((double)sp.ps[h], lsh));
    return v;
}

}  // namespace jhtb
