// fmm.cu — fast many-body (2-D FMM) on the device.
#include "fast.cuh"

namespace d3 {

void fmm_free(FastScratch &s) { s.fmm = nullptr; }

int fmm_run(FastScratch &s, TreeDev &t, const NodeArrays &a, const double *strengths,
            const FmmParams &p, const double *seed, uint32_t *status, cudaStream_t st) {
  return -3;
}

}  // namespace d3
