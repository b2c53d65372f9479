// Mixed-precision Laplace M2L on the sm_100a tensor cores (tcgen05, split
// TF32 products in FP32 in tensor memory, summed in registers).
#pragma once
#include "lap_common.cuh"

namespace b2 {

// M2L targets (boxes of levels >= 2 with list-2 boxes and evaluation
// points, sorted by list-2 length and interleaved into super-tiles of
// 128/ND x T targets) and their list-2 entries: the input of the
// tensor-core kernel.
struct M2LPairs {
  DBuf<int> tstart;                 // ntgt + 1 offsets into ent
  DBuf<int2> ent;                   // (source | offset index << 26, last-entry mark)
  DBuf<float> tab;                  // G (TF32 hi, lo) and the per-offset tables
  DBuf<unsigned long long> steps;   // steps of all super-tiles (tensor-core work)
  DBuf<int> info;                   // device counts: targets, super-tile size T, entries
  int n = 0;                        // candidate boxes (the arrays' size); 0: nothing to do
  int P = 0;
  bool usable = false;  // false: box indices do not fit the packed format or P too large
};

// Builds L for boxes [first, first+n) (P coefficients; chunk = densities of
// the main chunk, which sets the rows of a tile) without waiting on the
// host: counts stay on the device.  first may be RANGE_FROM2 (boxes of
// levels >= 2 from the tree's device level table, n = their upper bound).
void m2l_tc_build(M2LPairs& L, const lapk::TV& t, int first, int n, int nboxes, int P, int chunk,
                  cudaStream_t st);

// True when the tensor-core M2L supports P (expansion length).
bool m2l_tc_supported(int P);
// Coefficients per (box, density) of the FP32 multipole copy (P rounded up
// to a multiple of 4; the entries beyond P are zero).
int m2l_kh(int P);

// float2 elements of the FP32 multipole scratch for ND densities.
long m2l_tc_scratch(const M2LPairs& L, int nboxes, int ND);

// Enqueues the M2L contributions of all list-2 boxes into lo (FP64,
// [box][P][ND]) on st without synchronising (capturable in a CUDA graph).
// mp32: scratch of nmp32 >= m2l_tc_scratch() float2 for the FP32 copy of mp;
// boxsize: nlev (<= 64) box sizes by level.  A bounded wait for the tensor
// cores that gives up sets *err_dev to 1 (the caller reports IER_TIMEOUT
// after synchronising).
int m2l_tc_run(int ND, const M2LPairs& L, const double2* mp, float2* mp32, long nmp32, int nboxes,
               const TreeCtl* ctl, double2* lo, const double* boxsize, int nlev, int* err_dev, cudaStream_t st);

// Probe of the tensor-core tile path: D = A B^T for a 128 x K (A) and an
// N x K (B) FP32 matrix (row-major, device pointers), K in {8,16,24,32},
// N in {16,32}, with the same shared-memory layouts, split-TF32 products and
// tensor-memory read-back as the M2L kernel.  D is 128 x N row-major.
int tc_gemm_probe(const float* A, const float* B, int K, int N, float* D, cudaStream_t st);

}  // namespace b2
