// mlp.cuh — the learned correction's network: sizes, parameter layout and
// the tensor-core inference used by the fast many-body force's learned form.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace d3 {

constexpr int MLP_IN = 12, MLP_H = 64, MLP_OUT = 2;
// offsets in the parameter vector (weights [out][in], FP32 master copy)
constexpr int P_W1 = 0;
constexpr int P_B1 = P_W1 + MLP_H * MLP_IN;
constexpr int P_W2 = P_B1 + MLP_H;
constexpr int P_B2 = P_W2 + MLP_H * MLP_H;
constexpr int P_W3 = P_B2 + MLP_H;
constexpr int P_B3 = P_W3 + MLP_OUT * MLP_H;
constexpr int MLP_PARAMS = P_B3 + MLP_OUT;  // 5122

// y (n x 2) = MLP(x (n x 12)) on the tensor cores; device pointers; a failed
// wait sets ST_WAIT_TIMEOUT in *err_flag. Returns 0, or -1 if the launch failed.
int mlp_infer_tc(const float *x, uint32_t n, const float *params, float *y, uint32_t *err_flag,
                 cudaStream_t st);

}  // namespace d3
