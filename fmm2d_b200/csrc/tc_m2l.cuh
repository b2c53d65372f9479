// Mixed-precision Laplace M2L on the sm_100a tensor cores (tcgen05, TF32
// split products accumulated in FP32 in tensor memory).
#pragma once
#include "lap_common.cuh"

namespace b2 {

// Flattened list-2 pairs of all boxes of levels >= 2 that have evaluation
// points, ordered by target box:
// (target | level << 26, source | offset_index << 26).
struct M2LPairs {
  DBuf<int2> pairs;
  long npairs = 0;
  bool usable = false;  // false: box indices do not fit the packed format
};

void m2l_tc_build_pairs(M2LPairs& L, const lapk::TV& t, int first, int n, int nboxes,
                        cudaStream_t st);

// True when the tensor-core M2L supports P (expansion length).
bool m2l_tc_supported(int P);

// Enqueues the M2L contributions of all pairs into lo (FP64, [box][P][ND])
// on st without synchronising (capturable in a CUDA graph).
// utab/lgtab: (1/o)^k and log|o| tables of the 7x7 integer offsets; nlev:
// number of tree levels (entries of t.boxsize that are read), <= 64; mp32:
// scratch of nmp = nboxes * P * ND float2 for the FP32 copy of mp.  A bounded
// wait for the tensor cores that gives up sets *err_dev to 1 (the caller
// reports IER_TIMEOUT after synchronising).
int m2l_tc_run(int ND, const lapk::TV& t, const M2LPairs& L, int P, const double* binom,
               const float2* utab, const float* lgtab, const double2* mp, float2* mp32,
               long nmp, double2* lo, int nlev, int* err_dev, cudaStream_t st);

// Probe of the tensor-core tile path: D = A B^T for a 128 x K (A) and an
// N x K (B) FP32 matrix (row-major, device pointers), K in {8,16,24,32},
// N in {16,32}, with the same shared-memory layouts, split-TF32 products and
// tensor-memory read-back as the M2L kernel.  D is 128 x N row-major.
int tc_gemm_probe(const float* A, const float* B, int K, int N, float* D, cudaStream_t st);

}  // namespace b2
