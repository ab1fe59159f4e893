/*
 * gen_runtime.cuh — what the CUDA C emitted from MOD files (mind_b200.nmodl) runs on.
 *
 *   MindGenRow   one instance of a generated mechanism: its fields as columns of one
 *                allocation (column k of row r at cols[k * rows + r], the column-major
 *                data[row, field] of the reference, src/model/utils/build.jl:96-101) and
 *                the runtime inputs v, t, dt and celsius of the phase being run.
 *   MindAffine   the value and own-state coefficient of a cnexp right-hand side, with the
 *                arithmetic of the reference's AffineRate (src/compiler/codegen.jl:503-516).
 *   mind_exponential_factor  (e^x - 1)/x with its series below |x| = 1e-7 (codegen.jl:487-493).
 *   mind_gen_index  an array index truncated toward zero and clamped into the array.
 */
#pragma once

#include "mind_math.h"

namespace mind {

struct MindGenRow {
    double *cols;
    int64_t rows;
    int64_t row;
    double v, t, dt, celsius;
    __device__ __forceinline__ double &at(int k) const { return cols[(int64_t)k * rows + row]; }
};

struct MindAffine {
    double v, c;
};
__device__ __forceinline__ MindAffine operator+(MindAffine a, MindAffine b) { return {a.v + b.v, a.c + b.c}; }
__device__ __forceinline__ MindAffine operator-(MindAffine a, MindAffine b) { return {a.v - b.v, a.c - b.c}; }
__device__ __forceinline__ MindAffine operator-(MindAffine a) { return {-a.v, -a.c}; }
__device__ __forceinline__ MindAffine operator*(MindAffine a, MindAffine b) {
    return {a.v * b.v, a.c * b.v + a.v * b.c};
}
__device__ __forceinline__ MindAffine operator/(MindAffine a, MindAffine b) {
    return {a.v / b.v, (a.c - a.v / b.v * b.c) / b.v};
}

__device__ __forceinline__ double mind_exponential_factor(double x) {
    if (fabs(x) < 1.0e-7) return 1.0 + x * (0.5 + x * (1.0 / 6.0 + x / 24.0));
    return expm1(x) / x;
}

__device__ __forceinline__ int mind_gen_index(double x, int extent) {
    const double k = trunc(x);
    if (!(k >= 0.0)) return 0;
    return k >= (double)extent ? extent - 1 : (int)k;
}

}  // namespace mind
