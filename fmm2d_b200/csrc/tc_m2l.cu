// M2L of the mixed-precision Laplace FMM on the 5th-generation tensor cores.
//
// On scaled expansions (rscale = box size of the level, laprouts2d.f:1130-1244)
// the translation from a source box at integer offset o = (c_src - c_tgt)/bs
// (u = 1/o) factors into two diagonal scalings around one real matrix:
//     t_k = h_k (-u)^k,   y = G t,   L_i += u^i y_i  (i >= 1),
//     L_0 += y_0 + h_0 (log bs + log|o|),
// G_00 = 0, G_0k = 1 (k > 0), G_i0 = -1/i, G_ik = C(i+k-1, k-1).  G is the
// same for every offset and level, so the product y = G t of all pairs is
// one GEMM with a resident B operand; the scalings are FP32 complex
// multiplies by 49-entry tables in shared memory.
//
// Tiles of 128 rows (target box, density): step j takes every row's j-th
// list-2 source (a target has at most 27), so a tile runs <= 27 steps with
// one 128 x N x K MMA chain each (K = 2 KH real columns of t, real and
// imaginary parts interleaved; N = 2 KH rounded to 16).  Split TF32
// (cvt.rna on both parts): G t = A_hi B_hi + A_hi B_lo + A_lo B_hi with
// 22-bit operands, products in FP32 in tensor memory.
//
// Accumulation: the tensor cores round the FP32 sum of every MMA
// instruction toward zero.  Summed in place over a tile (27 offsets x 3
// passes x K/8 instructions) that bias reaches ~1e-5 of the locals, so each
// step has its own product in tensor memory, started by the two small terms
// (only the K/8 instructions of A_hi B_hi truncate at full magnitude), and
// the builders read it back (tcgen05.ld), scale it by u^i and sum the steps
// in FP32 registers with round-to-nearest: ~2e-7 relative, near a plain FP32
// M2L.
//
// Layouts: A (per stage, hi and lo) and B in shared memory use the canonical
// K-major layout without swizzle: element (r, k) of a tile with K columns
// sits at byte (r/8)*SBO + (k/4)*128 + (r%8)*16 + (k%4)*4, SBO = 32 K
// (8x16-byte core matrices, K-adjacent core matrices 128 bytes apart).
//
// Roles: builder warps (thread = one row x 4 coefficients) gather the
// source multipoles two steps ahead, scale and split them and write the A
// rows of a step into one of 4 shared-memory stages; one issuer thread waits
// for the stage (mbarrier) and issues the step's tcgen05.mma (M = 128, K = 8
// per instruction), whose commit releases the stage and its product.  At the
// end of a tile each builder thread adds its 4 coefficients to the FP64
// locals; each target row is written by exactly one thread.  Every wait on
// the tensor cores is bounded; on time-out the kernel records an error flag
// (reported as IER_TIMEOUT), frees its tensor memory and ends.
#include "tc_m2l.cuh"

#include <cub/cub.cuh>

#include "laplace.cuh"

namespace b2 {

namespace {

using namespace lapk;

constexpr int TC_ROWS = 128;
constexpr int TC_TMEM_COLS = 64;
constexpr long long TC_WAIT_CYCLES = 1LL << 31;  // ~1 s at the boost clock

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// UMMA shared-memory descriptor: start, leading and stride byte offsets (16-byte
// units), version 1 (sm_100), no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor: FP32 accumulator, TF32 A and B, both K-major.
__device__ __forceinline__ uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
          d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   mbar)
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count = 1) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

// Bounded wait for the given phase parity of the barrier: try_wait (which
// suspends the thread in hardware for a while) until the phase completes or
// about TC_WAIT_CYCLES SM clocks have passed.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > TC_WAIT_CYCLES) return false;
  }
}

// Non-blocking test of a barrier phase.
__device__ __forceinline__ bool mbar_test(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}

// The same bounded wait for threads that are usually early (the row builders
// run stages ahead of the tensor cores): each failed try backs off, so the
// waiting warps leave the issue slots to the MMA-issuing thread.
__device__ __forceinline__ bool mbar_wait_backoff(uint32_t mbar, uint32_t parity) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > TC_WAIT_CYCLES) return false;
    __nanosleep(256);
  }
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

// 16 consecutive FP32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(addr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
// 4 consecutive FP32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_ld4(uint32_t addr, float* v) {
  uint32_t r[4];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(addr)
               : "memory");
#pragma unroll
  for (int i = 0; i < 4; i++) v[i] = __uint_as_float(r[i]);
}
// 8 consecutive FP32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_ld8(uint32_t addr, float* v) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(addr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// byte offset of element (r, k) in a K-major tile with K columns
__device__ __forceinline__ uint32_t tile_off(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K * 32) + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

// Store 4 consecutive K values (k0 % 4 == 0) of row r as hi and lo tiles.
__device__ __forceinline__ void store_split4(char* hi, char* lo, int r, int k0, int K, float a0,
                                             float a1, float a2, float a3) {
  float h0 = tf32_rna(a0), h1 = tf32_rna(a1), h2 = tf32_rna(a2), h3 = tf32_rna(a3);
  uint32_t o = tile_off(r, k0, K);
  *reinterpret_cast<float4*>(hi + o) = make_float4(h0, h1, h2, h3);
  *reinterpret_cast<float4*>(lo + o) = make_float4(tf32_rna(a0 - h0), tf32_rna(a1 - h1),
                                                   tf32_rna(a2 - h2), tf32_rna(a3 - h3));
}

// Issue D (+)= A_hi B_hi + A_hi B_lo + A_lo B_hi over K / 8 steps.
__device__ __forceinline__ void issue_split_mma(uint32_t d_tmem, uint32_t a_hi, uint32_t a_lo,
                                                uint32_t b_hi, uint32_t b_lo, int K, uint32_t idesc) {
  const uint32_t sbo = (uint32_t)K * 32;
  for (int ks = 0; ks < K / 8; ks++) {
    uint32_t o = (uint32_t)ks * 256;
    uint64_t ah = umma_desc(a_hi + o, 128, sbo), al = umma_desc(a_lo + o, 128, sbo);
    uint64_t bh = umma_desc(b_hi + o, 128, sbo), bl = umma_desc(b_lo + o, 128, sbo);
    umma_tf32(d_tmem, ah, bh, idesc, ks > 0 ? 1u : 0u);
    umma_tf32(d_tmem, ah, bl, idesc, 1u);
    umma_tf32(d_tmem, al, bh, idesc, 1u);
  }
}

// ---------------------------------------------------------------------------
// M2L on the tensor cores
// ---------------------------------------------------------------------------
constexpr int OT_STAGES = 4;  // A stages in shared memory (power of 2)
constexpr int OT_DBUF = 8;    // product buffers in tensor memory (power of 2)
constexpr int NOFF = 64;      // table rows: offset index (ox + 3) * 7 + (oy + 3) < 49, rest zero
constexpr int NO_OFFSET = 63; // a row without a list-2 entry at this step (zero table row)

// Sizes and layouts for KH complex coefficients per row.  Columns of A and
// of the products interleave real and imaginary parts: A col 2k + c =
// (Re, Im) t_k, D col 2i + c = (Re, Im) y_i, D cols 2 KH, 2 KH + 1 = (Re, Im)
// S0 = t_0.  Two builder threads per row take C = KH / 2 coefficients each.
template <int KH>
struct OT {
  static constexpr int K = 2 * KH;                   // A columns
  static constexpr int N = (2 * KH + 2 + 15) / 16 * 16;  // product columns (+ S0)
  static constexpr int C = KH / 2;                   // coefficients per builder thread
  static constexpr int BUILDERS = 256;
  static constexpr int BWARPS = BUILDERS / 32;
  static constexpr int ISSUERS = OT_STAGES;          // MMA issuer warps (one thread each)
  static constexpr int THREADS = BUILDERS + 32 * ISSUERS;
  static constexpr uint32_t SA = 128u * K * 4;       // one A tile (hi or lo)
  static constexpr uint32_t SB = (uint32_t)N * K * 4;  // one B tile (hi or lo)
  static constexpr uint32_t A0 = 0;                  // A stages: [stage][hi, lo]
  static constexpr uint32_t B0 = OT_STAGES * 2 * SA; // G: [hi, lo]
  // offset tables, rows of KH + 2 float2: the 16-byte pad spreads the rows of
  // different offsets over all 8 groups of 16-byte shared-memory banks
  static constexpr int TS = KH + 2;
  static constexpr uint32_t UP = B0 + 2 * SB;        // float2 [NOFF][TS]: (-u)^k
  static constexpr uint32_t UO = UP + NOFF * TS * 8; // float2 [NOFF][TS]: u^i
  static constexpr uint32_t LGO = UO + NOFF * TS * 8;  // float [NOFF]: log|o|
  static constexpr uint32_t LGL = LGO + NOFF * 4;    // double [64]: log(box size) by level
  static constexpr uint32_t RING = LGL + 512;        // int [8][BUILDERS]: last-entry marks
  static constexpr uint32_t MISC = RING + 8 * BUILDERS * 4;  // mbarriers, tmem address, flags
  static constexpr uint32_t TOTAL = MISC + 128;
  // tensor memory: a ring of OT_DBUF products, step g in buffer g % OT_DBUF
  static constexpr uint32_t TMEM_USED = OT_DBUF * N;
  static constexpr uint32_t TMEM_COLS =
      TMEM_USED <= 128 ? 128 : (TMEM_USED <= 256 ? 256 : 512);
};

// float elements of the table image: G (hi, lo), then (-u)^k and u^i per
// offset index (float2), then log|o|.
__host__ __device__ constexpr long m2l_tab_floats(int KH) {
  return 2L * ((2 * KH + 2 + 15) / 16 * 16) * (2 * KH) + 4L * NOFF * (KH + 2) + NOFF;
}

// Round to TF32 (10 mantissa bits), to nearest with ties away from zero:
// add half a TF32 unit to the magnitude bits and clear the 13 low bits.
__device__ __forceinline__ float tf32_round(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

// The row's j-th list-2 entry (source | offset index << 26; none: NO_OFFSET << 26).
__device__ __forceinline__ unsigned ot_entry(int j, int ep, int ee, const int* __restrict__ ent) {
  return ep + j < ee ? (unsigned)ent[ep + j] : (unsigned)NO_OFFSET << 26;
}

// This thread's C coefficients of the multipole of entry e (zero for none).
template <int KH>
__device__ __forceinline__ void ot_fetch(unsigned e, const float4* __restrict__ mp32, int ND, int d,
                                         int part, float4 (&v)[KH / 4]) {
  constexpr int NV = KH / 4;  // float4 = 2 coefficients
  if ((e >> 26) != (unsigned)NO_OFFSET) {
    const float4* h = mp32 + ((size_t)(e & 0x3FFFFFFu) * ND + d) * (KH / 2) + NV * part;
#pragma unroll
    for (int m = 0; m < NV; m++) v[m] = h[m];
  } else {
#pragma unroll
    for (int m = 0; m < NV; m++) v[m] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

// 2C consecutive FP32 columns of this thread's tensor-memory lane (2C a
// multiple of 4, addr 4-column aligned), as 4-column loads.
template <int C>
__device__ __forceinline__ void tmem_ld_cols(uint32_t addr, float (&y)[2 * C]) {
#pragma unroll
  for (int m = 0; m < C / 2; m++) tmem_ld4(addr + 4 * m, y + 4 * m);
}

// One CTA per SM (persistent).  Rows are (target, density) pairs; 128 rows =
// R = 128/ND row groups.  A super-tile is R T consecutive targets of the
// order built by m2l_tc_build: row group q of the super-tile takes a
// contiguous run of about T targets (interleaved from the length-sorted
// order, so the runs have similar lengths) and walks their list-2 entries
// back to back, one per step.  ent: per entry (source | offset index << 26,
// target box | level << 26 on the last entry of a target, else -1); tstart:
// ntgt + 1 entry offsets; tab: the table image; mp32: FP32 multipoles
// [box][ND][KH] (zero beyond P); lo: FP64 locals [box][P][ND].
//
// Per step, with o the row's offset and u = 1/o:
//     t_k = h_k (-u)^k                        (builders, FP32)
//     y   = G t, S0 = t_0 = h_0               (tensor cores, split TF32)
//     L_i += u^i y_i,  L_0 += S0 log|o|       (builders, FP32 registers)
// and after the last entry of a target L_0 += log(bs) sum S0 and an FP64
// atomic add of the row's locals (each local has one writer).
//
// Pipeline: the builder warps (two threads per row, C coefficients each)
// write the A rows (hi, lo) of step g into shared-memory stage g % 4 once the
// MMAs of step g - 4 have released it (empty barrier, tcgen05.commit), and
// arrive on the stage's full barrier; the issuer thread then issues the
// step's MMAs into product buffer g % 8: A_hi B_lo (starting the product),
// A_lo B_hi, A_hi B_hi.  After the arrival the builders read back the
// product of step g - 4 (tcgen05.ld; its buffer is rewritten by step g + 4)
// and add it to their registers.  Loads run ahead: list entries three steps,
// multipoles two.  The tensor cores truncate each instruction's FP32 sum
// toward zero; with the two small terms first only the K/8 instructions of
// the main term truncate at full magnitude, and the steps are summed with
// round-to-nearest in registers.  The pipeline drains only at the end of a
// super-tile.
template <int KH>
__global__ void __launch_bounds__(OT<KH>::THREADS, 1)
    k_m2l_tc(const int* __restrict__ tstart, const int2* __restrict__ ent,
             const int* __restrict__ info, int ndsh, int P, const float4* __restrict__ tab,
             const double* __restrict__ boxsize, int nlev, const float4* __restrict__ mp32,
             double2* __restrict__ lo, int* __restrict__ err) {
  using L = OT<KH>;
  const int ntgt = info[0], T = info[1];
  constexpr int K = L::K, N = L::N, C = L::C, NV = KH / 4;
  extern __shared__ __align__(1024) char smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r = tid & 127, part = tid >> 7;
  const int ND = 1 << ndsh, R = 128 >> ndsh, d = r & (ND - 1), rg = r >> ndsh;
  uint32_t* misc = reinterpret_cast<uint32_t*>(smem + L::MISC);
  // full[OT_STAGES], empty[OT_STAGES] mbarriers, 8 bytes apart
  const uint32_t full0 = smem_u32(misc), empty0 = full0 + 8 * OT_STAGES;
  volatile uint32_t* s_taddr = misc + 4 * OT_STAGES;
  volatile int* s_fail = reinterpret_cast<volatile int*>(misc + 4 * OT_STAGES + 1);
  volatile int* s_wmax = reinterpret_cast<volatile int*>(misc + 4 * OT_STAGES + 2);  // [4]
  const float4* UP4 = reinterpret_cast<const float4*>(smem + L::UP);
  const float4* UO4 = reinterpret_cast<const float4*>(smem + L::UO);
  const float* LGO = reinterpret_cast<const float*>(smem + L::LGO);
  double* LGL = reinterpret_cast<double*>(smem + L::LGL);
  int* RING = reinterpret_cast<int*>(smem + L::RING);  // [8][BUILDERS]: last-entry marks

  {
    // G and the offset tables are contiguous in the image and in shared memory
    float4* dst = reinterpret_cast<float4*>(smem + L::B0);
    constexpr int nv = (int)(m2l_tab_floats(KH) / 4);
    for (int e = tid; e < nv; e += L::THREADS) dst[e] = tab[e];
  }
  for (int e = tid; e < 64; e += L::THREADS) LGL[e] = e < nlev ? log(boxsize[e]) : 0.0;
  if (tid == 0) {
    for (int q = 0; q < OT_STAGES; q++) {
      mbar_init(full0 + 8 * q, L::BWARPS);
      mbar_init(empty0 + 8 * q, 1);
    }
    *s_fail = 0;
  }
  __syncwarp();
  if (warp == 0) tmem_alloc(smem_u32((const void*)s_taddr), L::TMEM_COLS);
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t taddr = *s_taddr;
  const uint32_t lane_base = taddr + ((uint32_t)((warp & 3) * 32) << 16);
  const uint32_t sbase = smem_u32(smem);
  const long per_st = (long)R * T;
  const long nst = (ntgt + per_st - 1) / per_st;
  const bool builder = warp < L::BWARPS;
  // this thread's A columns 2 C part .. : C / 2 groups of 4, 128 bytes apart
  const uint32_t aoff = tile_off(r, 2 * C * part, K);
  uint32_t g = 0;  // steps of this CTA so far; stage g % OT_STAGES, buffer g % OT_DBUF

  for (long st = blockIdx.x; st < nst; st += gridDim.x) {
    // this row group's run of targets in the super-tile
    const long base = st * per_st;
    const int c = (int)min(per_st, (long)ntgt - base);
    const int q0 = c / R, rem = c % R;
    const int nr = builder ? q0 + (rg < rem ? 1 : 0) : 0;
    int ep = 0, ee = 0;
    if (nr > 0) {
      const long first = base + (long)rg * q0 + min(rg, rem);
      ep = tstart[first];
      ee = tstart[first + nr];
    }
    {
      const int m = __reduce_max_sync(~0u, ee - ep);
      if (lane == 0 && warp < 4) s_wmax[warp] = m;
    }
    __syncthreads();
    if (*s_fail) break;
    const uint32_t g0 = g;
    const uint32_t nsteps =
        (uint32_t)max(max(s_wmax[0], s_wmax[1]), max(s_wmax[2], s_wmax[3]));

    if (builder) {
      // this thread's coefficients i = C part + q of the current target's
      // locals, and (part 0) the sum of S0 for the level term
      float acc[2 * C], s0x = 0.f, s0y = 0.f;
#pragma unroll
      for (int q = 0; q < 2 * C; q++) acc[q] = 0.f;
      // offset index of step x in bits 6 (x % 8) .. + 5
      unsigned long long oring = 0;
      auto oring_get = [&](uint32_t x) { return (int)((oring >> (6 * (x % 8))) & 63u); };
      auto dcol = [&](uint32_t x) {
        return lane_base + (uint32_t)((x % OT_DBUF) * N + 2 * C * part);
      };
      // add the product of step x; after the last entry of a target, flush
      auto take = [&](uint32_t x) {
        float y[2 * C];
        tmem_ld_cols<C>(dcol(x), y);
        float z[4];
        if (part == 0) tmem_ld4(lane_base + (uint32_t)((x % OT_DBUF) * N + 2 * KH), z);
        tmem_wait_ld();
        const int op = oring_get(x);
        const float4* uo = UO4 + (op * L::TS + C * part) / 2;
#pragma unroll
        for (int m = 0; m < NV; m++) {
          const float4 w = uo[m];  // u^i for two coefficients
          acc[4 * m] = fmaf(y[4 * m], w.x, fmaf(-y[4 * m + 1], w.y, acc[4 * m]));
          acc[4 * m + 1] = fmaf(y[4 * m], w.y, fmaf(y[4 * m + 1], w.x, acc[4 * m + 1]));
          acc[4 * m + 2] = fmaf(y[4 * m + 2], w.z, fmaf(-y[4 * m + 3], w.w, acc[4 * m + 2]));
          acc[4 * m + 3] = fmaf(y[4 * m + 2], w.w, fmaf(y[4 * m + 3], w.z, acc[4 * m + 3]));
        }
        if (part == 0) {
          const float lg = LGO[op];
          acc[0] = fmaf(z[0], lg, acc[0]);
          acc[1] = fmaf(z[1], lg, acc[1]);
          s0x += z[0];
          s0y += z[1];
        }
        // -1: not the last entry of a target (a mark is box | level << 26 with
        // box < 2^26 - 1, never all ones)
        const int tb = RING[(x % 8) * L::BUILDERS + tid];
        if (tb != -1) {
          if (!*s_fail) {
            double* out = reinterpret_cast<double*>(
                lo + ((size_t)((unsigned)tb & 0x3FFFFFFu) * P + C * part) * ND + d);
#pragma unroll
            for (int q = 0; q < C; q++) {
              if (C * part + q < P) {
                double vx = (double)acc[2 * q], vy = (double)acc[2 * q + 1];
                if (q == 0 && part == 0) {
                  // the level term L_0 += log(bs) sum S0, in FP64
                  const double lg = LGL[(unsigned)tb >> 26];
                  vx += lg * (double)s0x;
                  vy += lg * (double)s0y;
                }
                atomicAdd(out + 2 * (size_t)q * ND, vx);
                atomicAdd(out + 2 * (size_t)q * ND + 1, vy);
              }
            }
          }
#pragma unroll
          for (int q = 0; q < 2 * C; q++) acc[q] = 0.f;
          s0x = s0y = 0.f;
        }
      };
      // Step j from the fetched entry (ecur, vcur).  The multipole of step
      // j + 2 (entry en, read one step earlier) goes to (ef, vf) and the entry
      // of step j + 3 to en, so no load waits for another.  The rows are
      // computed before the wait for the stage, so only the split, the
      // stores, the proxy fence and the arrival follow the release; the
      // product of step g - 4 is read after the arrival.
      const int2 none = make_int2(NO_OFFSET << 26, -1);
      auto entry = [&](uint32_t j) { return ep + (int)j < ee ? ent[ep + j] : none; };
      int2 en;
      auto body = [&](uint32_t j, int2 ecur, const float4 (&vcur)[NV], int2& ef,
                      float4 (&vf)[NV]) {
        ef = en;
        ot_fetch<KH>((unsigned)ef.x, mp32, ND, d, part, vf);
        en = entry(j + 3);
        const int s = (int)(g % OT_STAGES);
        const int oi = (int)((unsigned)ecur.x >> 26);
        // t = h (-u)^k
        float4 t[NV];
        {
          const float4* up = UP4 + (oi * L::TS + C * part) / 2;
#pragma unroll
          for (int m = 0; m < NV; m++) {
            const float4 w = up[m];  // (-u)^k for two coefficients
            const float4 h = vcur[m];
            t[m] = make_float4(h.x * w.x - h.y * w.y, h.x * w.y + h.y * w.x,
                               h.z * w.z - h.w * w.w, h.z * w.w + h.w * w.z);
          }
        }
        RING[(g % 8) * L::BUILDERS + tid] = ecur.y;
        if (g >= OT_STAGES && !*s_fail) {
          if (!mbar_wait_backoff(empty0 + 8 * s, (g / OT_STAGES - 1) & 1)) *s_fail = 1;
          tc_fence_after();
        }
        // TF32 hi (rounded) and lo (the MMA keeps its leading 11 bits)
        {
          char* A = smem + L::A0 + (size_t)s * 2 * L::SA + aoff;
#pragma unroll
          for (int m = 0; m < NV; m++) {
            const float4 hi = make_float4(tf32_round(t[m].x), tf32_round(t[m].y),
                                          tf32_round(t[m].z), tf32_round(t[m].w));
            *reinterpret_cast<float4*>(A + 128 * m) = hi;
            *reinterpret_cast<float4*>(A + L::SA + 128 * m) =
                make_float4(t[m].x - hi.x, t[m].y - hi.y, t[m].z - hi.z, t[m].w - hi.w);
          }
        }
        // visible to the tensor cores, then published
        fence_async_smem();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(full0 + 8 * s);
        if (g >= g0 + OT_STAGES) take(g - OT_STAGES);
        oring = (oring & ~(63ull << (6 * (g % 8)))) | ((unsigned long long)oi << (6 * (g % 8)));
        ++g;
      };
      int2 e0 = entry(0), e1 = entry(1), e2;
      en = entry(2);
      float4 v0[NV], v1[NV], v2[NV];
      ot_fetch<KH>((unsigned)e0.x, mp32, ND, d, part, v0);
      ot_fetch<KH>((unsigned)e1.x, mp32, ND, d, part, v1);
      for (uint32_t j = 0; j < nsteps; j += 3) {
        body(j, e0, v0, e2, v2);
        if (j + 1 < nsteps) body(j + 1, e1, v1, e0, v0);
        if (j + 2 < nsteps) body(j + 2, e2, v2, e1, v1);
      }
      // the super-tile's last (up to 4) products, in order as their commits complete
      for (uint32_t x = g - min(nsteps, (uint32_t)OT_STAGES); x < g; x++) {
        if (!*s_fail && !mbar_wait(empty0 + 8 * (x % OT_STAGES), (x / OT_STAGES) & 1))
          *s_fail = 1;
        tc_fence_after();
        take(x);
      }
    } else if (lane == 0) {
      // MMA issuers: issuer w takes the steps g = w (mod OT_STAGES), i.e.
      // always stage w, so that the steps of OT_STAGES stages are issued
      // concurrently (one thread issues a tcgen05.mma only every ~150 SM
      // clocks; four threads together reach ~40-50).  Each commit covers the
      // issuing thread's own MMAs: the commit of step g releases stage
      // g % OT_STAGES and marks product g % OT_DBUF complete.
      const uint32_t w = (uint32_t)(warp - L::BWARPS);
      const uint32_t idesc = idesc_tf32(TC_ROWS, N);
      const uint64_t bh = umma_desc(sbase + L::B0, 128, (uint32_t)K * 32);
      const uint64_t bl = bh + (L::SB >> 4);
      bool fail = *s_fail != 0;
      const uint32_t first = g0 + ((w + OT_STAGES - g0 % OT_STAGES) % OT_STAGES);
      for (uint32_t x = first; x < g0 + nsteps; x += OT_STAGES) {
        const int s = (int)(x % OT_STAGES);
        if (!fail && !mbar_wait(full0 + 8 * s, (x / OT_STAGES) & 1)) fail = true;
        tc_fence_after();
        if (!fail) {
          const uint32_t dt = taddr + (uint32_t)((x % OT_DBUF) * N);
          // a K step of 8 columns advances a start address by 256 bytes
          // (16 in descriptor units)
          const uint64_t ah =
              umma_desc(sbase + L::A0 + (uint32_t)s * 2 * L::SA, 128, (uint32_t)K * 32);
          const uint64_t al = ah + (L::SA >> 4);
#pragma unroll
          for (int ks = 0; ks < K / 8; ks++)
            umma_tf32(dt, ah + 16 * ks, bl + 16 * ks, idesc, ks == 0 ? 0u : 1u);
#pragma unroll
          for (int ks = 0; ks < K / 8; ks++) umma_tf32(dt, al + 16 * ks, bh + 16 * ks, idesc, 1u);
#pragma unroll
          for (int ks = 0; ks < K / 8; ks++) umma_tf32(dt, ah + 16 * ks, bh + 16 * ks, idesc, 1u);
        }
        // the commit also releases the stage when nothing was issued
        umma_commit(empty0 + 8 * s);
      }
      if (fail) *s_fail = 1;
    }
    g = g0 + nsteps;
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  if (*s_fail && tid == 0) {
    // the tensor cores may still be working: one more bounded wait for the
    // last commit of every stage before the tensor memory is released
    for (uint32_t gl = g > OT_STAGES ? g - OT_STAGES : 0; gl < g; gl++)
      mbar_wait(empty0 + 8 * (gl % OT_STAGES), (gl / OT_STAGES) & 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(taddr, L::TMEM_COLS);
  if (tid == 0 && *s_fail) atomicExch(err, 1);
}

// Table image for KH coefficients (P used): G in the canonical K-major
// layout as TF32 hi and lo tiles (B[n][kc] = G_ik for n = 2i + c, kc = 2k + c:
// real G acting on Re and Im alike; rows 2 KH + c pick t_0), then (-u)^k and
// u^i per offset index and log|o| (FP32; zero rows for the indices that are
// not offsets).
// G_00 = 0, G_0k = 1, G_i0 = -1/i, G_ik = C(i+k-1, k-1).
__global__ void k_m2l_tab(int KH, int N, int P, const double* __restrict__ binom,
                          float* __restrict__ out) {
  const int K = 2 * KH;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < N * K) {
    const int n = e / K, kc = e % K;
    double v = 0.0;
    const int i = n >> 1, k = kc >> 1;
    if (n < 2 * KH && (n & 1) == (kc & 1) && i < P && k < P) {
      if (i == 0)
        v = k == 0 ? 0.0 : 1.0;
      else if (k == 0)
        v = -1.0 / i;
      else
        v = binom[(size_t)(i + k - 1) * BINOM_N + (k - 1)];
    } else if (kc < 2 && n == 2 * KH + kc) {
      v = 1.0;  // S0 = t_0 (rows 2 KH, 2 KH + 1; columns 0, 1)
    }
    const float hi = tf32_rna((float)v), lw = tf32_rna((float)(v - (double)hi));
    const uint32_t o = tile_off(n, kc, K) / 4;
    out[o] = hi;
    out[(size_t)N * K + o] = lw;
    return;
  }
  // tables: rows of TS = KH + 2 float2 (the last two are padding, zero)
  const int TS = KH + 2;
  const int f = e - N * K;
  if (f >= NOFF * TS) return;
  float2* up = reinterpret_cast<float2*>(out + 2L * N * K);
  float2* uo = up + NOFF * TS;
  float* lg = reinterpret_cast<float*>(uo + NOFF * TS);
  const int oi = f / TS, k = f % TS;
  if (k >= KH) {
    up[f] = uo[f] = make_float2(0.f, 0.f);
    return;
  }
  const int ox = oi / 7 - 3, oy = oi % 7 - 3;
  double2 p = make_double2(0.0, 0.0);
  double l = 0.0;
  if (oi < 49 && (ox != 0 || oy != 0)) {
    const double den = (double)ox * ox + (double)oy * oy;
    const double ur = ox / den, ui = -oy / den;  // u = 1/o
    p = make_double2(1.0, 0.0);
    for (int q = 0; q < k; q++) p = make_double2(p.x * ur - p.y * ui, p.x * ui + p.y * ur);
    l = 0.5 * log(den);
  }
  uo[f] = make_float2((float)p.x, (float)p.y);
  const double sg = (k & 1) ? -1.0 : 1.0;
  up[f] = make_float2((float)(sg * p.x), (float)(sg * p.y));
  if (k == 0) lg[oi] = (float)l;
}

// FP32 copy of one density chunk's multipoles, [box][ND][KH] (zero beyond P),
// two coefficients per thread; only the boxes the tree holds (its count read
// from the control block when there is one), grid-stride.
__global__ void k_mp_to_f32(const double2* __restrict__ mp, long nbox, const TreeCtl* ctl, int P,
                            int ND, int KH, float4* __restrict__ out) {
  const long nb = ctl ? min((long)ctl->nboxes, nbox) : nbox;
  const int KH2 = KH >> 1;
  const long total = nb * ND * KH2;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const int k = (int)(e % KH2) * 2;
    const long bd = e / KH2;
    const int d = (int)(bd % ND);
    const long box = bd / ND;
    const double2* src = mp + ((size_t)box * P + k) * ND + d;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (k < P) {
      const double2 x = src[0];
      v.x = (float)x.x;
      v.y = (float)x.y;
    }
    if (k + 1 < P) {
      const double2 x = src[ND];
      v.z = (float)x.x;
      v.w = (float)x.y;
    }
    out[e] = v;
  }
}

__global__ void __launch_bounds__(128, 1)
    k_tc_gemm_probe(const float* __restrict__ Ag, const float* __restrict__ Bg, int K, int N,
                    float* __restrict__ Dg, int* __restrict__ err) {
  extern __shared__ __align__(1024) char smem[];
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t SA = 128u * K * 4, SB = (uint32_t)N * K * 4;
  char* A = smem;
  char* B = smem + 2 * SA;
  uint32_t* misc = reinterpret_cast<uint32_t*>(smem + 2 * SA + 2 * SB);
  const uint32_t mbar = smem_u32(misc);
  volatile uint32_t* s_taddr = misc + 2;
  for (int k0 = 0; k0 < K; k0 += 4) {
    const float* a = Ag + (size_t)tid * K + k0;
    store_split4(A, A + SA, tid, k0, K, a[0], a[1], a[2], a[3]);
  }
  for (int e = tid; e < N * (K / 4); e += blockDim.x) {
    int n = e / (K / 4), k0 = (e % (K / 4)) * 4;
    const float* b = Bg + (size_t)n * K + k0;
    store_split4(B, B + SB, n, k0, K, b[0], b[1], b[2], b[3]);
  }
  if (tid == 0) mbar_init(mbar);
  __syncwarp();
  if (warp == 0) tmem_alloc(smem_u32((const void*)s_taddr), TC_TMEM_COLS);
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t taddr = *s_taddr;
  if (tid == 0) {
    issue_split_mma(taddr, smem_u32(A), smem_u32(A) + SA, smem_u32(B), smem_u32(B) + SB, K,
                    idesc_tf32(TC_ROWS, N));
    umma_commit(mbar);
  }
  bool ok = mbar_wait(mbar, 0);
  tc_fence_after();
  float y[32];
  const uint32_t lane_addr = taddr + ((uint32_t)(warp * 32) << 16);
  tmem_ld16(lane_addr, y);
  if (N > 16) tmem_ld16(lane_addr + 16, y + 16);
  tmem_wait_ld();
  for (int n = 0; n < N; n++) Dg[(size_t)tid * N + n] = ok ? y[n] : 0.f;
  if (!ok) atomicExch(err, 1);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(taddr, TC_TMEM_COLS);
}

// Candidate i of the target range (a box of level >= 2 with list-2 boxes
// and evaluation points); the range may come from the device level table,
// and n (the scan length) may exceed it.
__global__ void k_m2l_flag(TV t, int first, int n, int* __restrict__ flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int f = first, nn = n;
  resolve_range(t, f, nn);
  const int b = f + i;
  flag[i] = (i < nn && t.has_eval_pts(b) && t.nl2[b] > 0) ? 1 : 0;
}

// Target count (info[0]) and super-tile size T (info[1]): about four
// super-tiles per SM for R rows.
__global__ void k_m2l_info(const int* __restrict__ tix, const int* __restrict__ flag, int n,
                           int R, int nsm, int* __restrict__ info) {
  const int ntgt = n > 0 ? tix[n - 1] + flag[n - 1] : 0;
  info[0] = ntgt;
  const long rows = ((long)ntgt + R - 1) / R;
  info[1] = (int)max(1L, (rows + 4L * nsm - 1) / (4L * nsm));
}

// Compact the targets with their list-2 length as the sort key: a tile runs
// as many steps as its longest list, so tiles of equal lengths keep every
// row busy.  Non-targets keep key 31 (set beforehand) and sort last.
__global__ void k_m2l_compact(TV t, int first, int n, const int* __restrict__ flag,
                              const int* __restrict__ tix, int* __restrict__ key,
                              int* __restrict__ box) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !flag[i]) return;
  int f = first, nn = n;
  resolve_range(t, f, nn);
  const int b = f + i;
  key[tix[i]] = t.nl2[b];
  box[tix[i]] = b;
}

__global__ void k_m2l_count(TV t, const int* __restrict__ box, int n,
                            const int* __restrict__ info, int* __restrict__ cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) cnt[i] = i < info[0] ? t.nl2[box[i]] : 0;
}

// Entry count (info[2]) and the closing offset tstart[ntgt].
__global__ void k_m2l_total(const int* __restrict__ offs, const int* __restrict__ cnt,
                            int* __restrict__ info, int* __restrict__ tstart) {
  const int ntgt = info[0];
  const int np = ntgt > 0 ? offs[ntgt - 1] + cnt[ntgt - 1] : 0;
  info[2] = np;
  tstart[ntgt] = np;
}

// Target boxes in kernel order and their list-2 entries, sorted by offset
// index: (source | offset index << 26, target box | level << 26 on the last
// entry of a target, else -1).  The kernel accepts any order; sorted, the
// rows of neighbouring targets (same child position) tend to take the same
// offset in the same step, so their table loads coincide (2.13 against
// 2.25 ms for the M2L at 4M points in list order).
__global__ void __launch_bounds__(128) k_m2l_fill(TV t, const int* __restrict__ box,
                                                  const int* __restrict__ info,
                                                  const int* __restrict__ cnt,
                                                  const int* __restrict__ offs,
                                                  int* __restrict__ tstart,
                                                  int2* __restrict__ ent) {
  // a target has at most one list-2 box per offset index (< 49): each thread
  // places its entries in its own 49 slots and emits them in index order
  __shared__ int slot[49][128];
  const int ti = blockIdx.x * blockDim.x + threadIdx.x;
  if (ti >= info[0]) return;
  const int b = box[ti], n2 = cnt[ti];
  const double2 cb = t.center[b];
  const double rinv = 1.0 / t.boxsize[t.level[b]];
  unsigned long long mask = 0;
  for (int e = 0; e < n2; e++) {
    const int jb = t.l2[(size_t)MNLIST2 * b + e];
    const double2 cj = t.center[jb];
    const int ox = __double2int_rn((cj.x - cb.x) * rinv), oy = __double2int_rn((cj.y - cb.y) * rinv);
    const int oi = (ox + 3) * 7 + (oy + 3);
    slot[oi][threadIdx.x] = jb;
    mask |= 1ull << oi;
  }
  const int o = offs[ti];
  const int tb = (int)((unsigned)b | ((unsigned)t.level[b] << 26));
  for (int e = 0; mask; e++) {
    const int oi = __ffsll((long long)mask) - 1;
    mask &= mask - 1;
    ent[o + e] = make_int2((int)((unsigned)slot[oi][threadIdx.x] | ((unsigned)oi << 26)),
                           mask ? -1 : tb);
  }
  tstart[ti] = o;
}

// Kernel order of the length-sorted targets: super-tiles of R T targets, in
// which row group q takes a contiguous run of the targets q, q + R, q + 2R,
// ... of the super-tile (runs of similar total length).
__global__ void k_m2l_perm(const int* __restrict__ sbox, const int* __restrict__ info, int R,
                           int* __restrict__ pbox) {
  const int ntgt = info[0], T = info[1];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ntgt) return;
  const long per = (long)R * T, base = i / per * per;
  const int ip = (int)(i - base);
  const int c = (int)min(per, (long)ntgt - base), q0 = c / R, rem = c % R;
  const int rg = ip % R, k = ip / R;
  pbox[base + (long)rg * q0 + min(rg, rem) + k] = sbox[i];
}

// Steps of all super-tiles (the issued tensor-core work): the longest run
// of list-2 entries over the row groups of each super-tile.
__global__ void k_m2l_steps(const int* __restrict__ tstart, const int* __restrict__ info, int R,
                            unsigned long long* __restrict__ out) {
  const long ntgt = info[0];
  const int T = info[1];
  const long stl = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long per = (long)R * T, base = stl * per;
  if (base >= ntgt) return;
  const int c = (int)min(per, ntgt - base), q0 = c / R, rem = c % R;
  int m = 0;
  for (int rg = 0; rg < R; rg++) {
    const int nr = q0 + (rg < rem ? 1 : 0);
    if (nr == 0) continue;
    const long first = base + (long)rg * q0 + min(rg, rem);
    m = max(m, tstart[first + nr] - tstart[first]);
  }
  atomicAdd(out, (unsigned long long)m);
}

}  // namespace

int m2l_kh(int P) { return (P + 3) / 4 * 4; }

bool m2l_tc_supported(int P) { return P >= 2 && P <= 20; }

void m2l_tc_build(M2LPairs& L, const TV& t, int first, int n, int nboxes, int P, int chunk,
                  cudaStream_t st) {
  L.P = P;
  L.n = 0;
  L.usable = nboxes < (1 << 26) && m2l_tc_supported(P);
  if (!L.usable || n <= 0) return;
  L.n = n;
  // every count stays on the device (info: targets, super-tile size,
  // entries); the arrays are sized for n candidates
  L.info.alloc(4, st);
  L.info.zero(4);
  DBuf<int> flag(st), tix(st);
  flag.alloc(n, st);
  tix.alloc(n, st);
  k_m2l_flag<<<ceil_div(n, 256), 256, 0, st>>>(t, first, n, flag.p);
  B2_LAUNCH_CHECK();
  size_t tb = 0;
  B2_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, tb, flag.p, tix.p, n, st));
  DBuf<char> tmp(st);
  tmp.alloc(tb, st);
  B2_CHECK(cub::DeviceScan::ExclusiveSum(tmp.p, tb, flag.p, tix.p, n, st));
  int dev = 0, nsm = 148;
  B2_CHECK(cudaGetDevice(&dev));
  B2_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int R = 128 / chunk;
  k_m2l_info<<<1, 1, 0, st>>>(tix.p, flag.p, n, R, nsm, L.info.p);
  B2_LAUNCH_CHECK();
  // targets sorted by list-2 length (non-targets: key 31, sorted last)
  DBuf<int> key(st), box(st), skey(st), sbox(st), cnt(st), offs(st);
  key.alloc(n, st);
  box.alloc(n, st);
  skey.alloc(n, st);
  sbox.alloc(n, st);
  key.fill_bytes(0x1f, n);
  box.fill_bytes(0xff, n);
  k_m2l_compact<<<ceil_div(n, 256), 256, 0, st>>>(t, first, n, flag.p, tix.p, key.p, box.p);
  B2_LAUNCH_CHECK();
  size_t tb2 = 0;
  // list lengths are <= MNLIST2 < 31: 5 key bits (stable: box order inside a length)
  static_assert(MNLIST2 < 31, "list-2 length key");
  B2_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, tb2, key.p, skey.p, box.p, sbox.p, n, 0, 5,
                                           st));
  DBuf<char> tmp2(st);
  tmp2.alloc(tb2, st);
  B2_CHECK(cub::DeviceRadixSort::SortPairs(tmp2.p, tb2, key.p, skey.p, box.p, sbox.p, n, 0, 5,
                                           st));
  DBuf<int> pbox(st);
  pbox.alloc(n, st);
  k_m2l_perm<<<ceil_div(n, 256), 256, 0, st>>>(sbox.p, L.info.p, R, pbox.p);
  B2_LAUNCH_CHECK();
  cnt.alloc(n, st);
  offs.alloc(n, st);
  k_m2l_count<<<ceil_div(n, 256), 256, 0, st>>>(t, pbox.p, n, L.info.p, cnt.p);
  B2_LAUNCH_CHECK();
  size_t tb3 = 0;
  B2_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, tb3, cnt.p, offs.p, n, st));
  DBuf<char> tmp3(st);
  tmp3.alloc(tb3, st);
  B2_CHECK(cub::DeviceScan::ExclusiveSum(tmp3.p, tb3, cnt.p, offs.p, n, st));
  L.tstart.alloc((size_t)n + 1, st);
  L.ent.alloc((size_t)MNLIST2 * n, st);
  k_m2l_total<<<1, 1, 0, st>>>(offs.p, cnt.p, L.info.p, L.tstart.p);
  B2_LAUNCH_CHECK();
  k_m2l_fill<<<ceil_div(n, 128), 128, 0, st>>>(t, pbox.p, L.info.p, cnt.p, offs.p, L.tstart.p,
                                               L.ent.p);
  B2_LAUNCH_CHECK();
  const int KH = m2l_kh(P), K = 2 * KH, N = (2 * KH + 2 + 15) / 16 * 16;
  L.tab.alloc(m2l_tab_floats(KH), st);
  k_m2l_tab<<<ceil_div(N * K + NOFF * (KH + 2), 256), 256, 0, st>>>(KH, N, P, device_binomials(),
                                                               L.tab.p);
  B2_LAUNCH_CHECK();
  L.steps.alloc(1, st);
  L.steps.zero(1);
  k_m2l_steps<<<ceil_div(n / R + 1, 128), 128, 0, st>>>(L.tstart.p, L.info.p, R, L.steps.p);
  B2_LAUNCH_CHECK();
  // the temporaries above are freed (stream-ordered) when this returns
}

long m2l_tc_scratch(const M2LPairs& L, int nboxes, int ND) {
  return (long)nboxes * ND * m2l_kh(L.P);
}

int m2l_tc_run(int ND, const M2LPairs& L, const double2* mp, float2* mp32, long nmp32, int nboxes,
               const TreeCtl* ctl, double2* lo, const double* boxsize, int nlev, int* err_dev, cudaStream_t st) {
  if (L.n == 0) return IER_OK;
  const int P = L.P;
  if (nlev > 64 || !m2l_tc_supported(P) || !(ND == 1 || ND == 2 || ND == 4 || ND == 8))
    return IER_BADARG;
  if (nmp32 < m2l_tc_scratch(L, nboxes, ND)) return IER_BADARG;
  const int KH = m2l_kh(P);
  const int ndsh = ND == 8 ? 3 : (ND == 4 ? 2 : (ND == 2 ? 1 : 0));
  int dev = 0, nsm = 148;
  B2_CHECK(cudaGetDevice(&dev));
  B2_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const long nconv = (long)nboxes * ND * (KH / 2);
  k_mp_to_f32<<<(int)std::min<long>(ceil_div(nconv, 256), (long)nsm * 8), 256, 0, st>>>(
      mp, nboxes, ctl, P, ND, KH, reinterpret_cast<float4*>(mp32));
  B2_LAUNCH_CHECK();
  auto launch = [&](auto kern, uint32_t total, uint32_t tmem_cols, int threads) {
    // CTAs that can share an SM (tensor-memory columns and shared memory);
    // the shared memory request keeps more from being resident (a tensor
    // memory allocation would wait)
    const int per_sm = std::max(1, std::min(512 / (int)tmem_cols, 232448 / (int)(total + 1024)));
    const size_t sm = std::max<size_t>(total, (size_t)(233472 / (per_sm + 1)) + 1024);
    set_smem_attr(kern, sm);
    // persistent: the CTAs take the super-tiles (counted on the device) in turn
    const int grid = (int)std::min<long>((long)L.n, (long)nsm * per_sm);
    kern<<<grid, threads, sm, st>>>(L.tstart.p, L.ent.p, L.info.p, ndsh, P,
                                    reinterpret_cast<const float4*>(L.tab.p), boxsize, nlev,
                                    reinterpret_cast<const float4*>(mp32), lo, err_dev);
    B2_LAUNCH_CHECK();
  };
#define B2_OT(KHV) \
  launch(k_m2l_tc<KHV>, OT<KHV>::TOTAL, OT<KHV>::TMEM_COLS, OT<KHV>::THREADS)
  switch (KH) {
    case 4: B2_OT(4); break;
    case 8: B2_OT(8); break;
    case 12: B2_OT(12); break;
    case 16: B2_OT(16); break;
    default: B2_OT(20); break;
  }
#undef B2_OT
  return IER_OK;
}

int tc_gemm_probe(const float* A, const float* B, int K, int N, float* D, cudaStream_t st) {
  if (!(K == 8 || K == 16 || K == 24 || K == 32) || !(N == 16 || N == 32)) return IER_BADARG;
  size_t sm = 2 * 128 * K * 4 + 2 * N * K * 4 + 32;
  DBuf<int> err(st);
  err.alloc(1, st);
  err.zero(1);
  set_smem_attr(k_tc_gemm_probe, sm);
  k_tc_gemm_probe<<<1, 128, sm, st>>>(A, B, K, N, D, err.p);
  B2_LAUNCH_CHECK();
  int* h = pinned_ints(1);
  B2_CHECK(cudaMemcpyAsync(h, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  B2_CHECK(cudaStreamSynchronize(st));
  return h[0] ? IER_TIMEOUT : IER_OK;
}

}  // namespace b2
