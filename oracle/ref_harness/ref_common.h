// ref_common.h -- shared declarations of the reference-kernel harness.
//
// TEST INFRASTRUCTURE ONLY. The harness compiles gilbs10/OpenFusion's own CUDA
// kernel sources (included from the reference tree at build time, never
// copied) into oracle/_ref/libref_kernels.so, so that the oracle can be pinned
// against outputs of the reference itself on the same inputs. The reference's
// compile-time constants are used as they are (Constants.h: VOLUME_SIZE 512,
// worldVolume 1024 mm, TRUNCATION 10 mm, MAX_WEIGHT 120).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

extern "C" {
typedef struct ref_cam {
  int32_t w, h;
  float fx, fy, cx, cy;   // m_intrinsic
  float ifx, ify, icx, icy;  // m_invIntrinsic (inverse K entries, CameraFromFile.cpp:42-51)
  float dmin, dmax;
} ref_cam;
}

#define REF_TRY(x)                                   \
  do {                                               \
    cudaError_t e_ = (x);                            \
    if (e_ != cudaSuccess) return (int)e_;           \
  } while (0)
