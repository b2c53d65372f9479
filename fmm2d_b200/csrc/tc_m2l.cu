// M2L of the mixed-precision Laplace FMM on the 5th-generation tensor cores.
//
// On scaled expansions (rscale = box size of the level, laprouts2d.f:1130-1244)
// the translation from a source box at integer offset o = (c_src - c_tgt)/bs
// is a complex matrix of the offset alone,
//     L_i += sum_k T_o[i][k] h_k,     T_o[i][k] = u^i G_ik (-u)^k,  u = 1/o,
// G_0k = 1 (k > 0), G_i0 = -1/i, G_ik = C(i+k-1, k-1), T_o[0][0] = log|o|,
// plus the level term L_0 += log(bs) h_0.  A target box has at most one
// list-2 source per offset, so the M2L of a tile of 128 rows (target box,
// density) is a sum over the <= 40 offsets of one GEMM each,
//     Y[rows, :] += A_o[rows, :] B_o^T,
// with A_o the multipole of every row's source at offset o (a zero row where
// the target has none).  The accumulator stays in tensor memory across the
// offsets and the result is written once per target: no per-pair scaling, no
// reduction over pairs and no atomics.
//
// The 40 offsets are images of 7 base offsets b (2,0) (2,1) (2,2) (3,0)
// (3,1) (3,2) (3,3) under the 8 symmetries of the square, o = w b or
// o = w conj(b) with w = i^m.  With u = conj(w) u_b (or conj(w) conj(u_b)),
//     T_o h = conj(w)^i (T'_b h'),   h'_k = conj(w)^k h_k,   T'_b = T_b or conj(T_b):
// the row builders apply the input phases (exact swaps and sign changes of
// the FP32 values), each rotation class m accumulates in its own
// tensor-memory columns, and the epilogue applies the output phases and sums
// the 4 classes.  The 14 operators T_b, conj(T_b) (TF32 hi + lo) stay
// resident in shared memory for the whole kernel.
//
// Complex products as real GEMMs, real and imaginary parts interleaved:
// A row = (Re, Im) h'_0 .. h'_{KH-1} (K = 2 KH), Y row = (Re, Im) L_0 ..
// L_{KH-1}, then (Re, Im) S0 with S0 = sum of h_0 over the row's sources
// (for the log(bs) term), B = 2x2 blocks [[Re T, -Im T], [Im T, Re T]] plus
// the two S0 rows.  Split TF32 (cvt.rna): A B = A_hi B_hi + A_hi B_lo +
// A_lo B_hi, FP32-level accuracy, accumulated in FP32 in tensor memory.
//
// B tiles in shared memory use the canonical K-major layout without
// swizzle: element (r, k) of a tile with K columns sits at byte
// (r/8)*SBO + (k/4)*128 + (r%8)*16 + (k%4)*4, SBO = 32 K (8x16-byte core
// matrices, K-adjacent core matrices 128 bytes apart).  The A rows live in
// tensor memory (lane = row), written by the builders with tcgen05.st.
//
// Roles: builder warps (thread = one row x 4 coefficients) gather the
// source multipoles two offset steps ahead, apply the phases, split and
// write the rows of a step into one of 4 tensor-memory stages; one issuer
// thread waits for the stage (mbarrier) and issues the step's tcgen05.mma
// (M = 128, N = 2 KH + 2 rounded to 16, K = 8 per instruction, A from
// tensor memory, B from shared memory), whose commit releases the stage.
// Targets are grouped by their position in the parent box, which fixes the
// set of offsets a target can have (at most 27 of the 40), so a tile runs
// few offset steps.  At the end of a tile every builder thread reads back
// its coefficients of the 4 class accumulators (tcgen05.ld) and adds them to
// the FP64 locals; each target row is written by exactly one thread.
// Every wait on the tensor cores is bounded; on time-out the kernel records
// an error flag (reported as IER_TIMEOUT), frees its tensor memory and ends.
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
  *reinterpret_cast<float4*>(lo + o) = make_float4(a0 - h0, a1 - h1, a2 - h2, a3 - h3);
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
// offset-accumulating M2L
// ---------------------------------------------------------------------------
constexpr int NBASE = 7;
constexpr int NBMAT = 2 * NBASE;  // the base operators and their conjugates
constexpr int OT_STAGES = 4;      // A stages in tensor memory (power of 2)
__host__ __device__ constexpr int base_ox(int b) { return b < 3 ? 2 : 3; }
__host__ __device__ constexpr int base_oy(int b) { return b < 3 ? b : b - 3; }

// Sizes and layouts for KH complex coefficients per row.  Columns of A and
// of the accumulators interleave real and imaginary parts: A col 2k + c =
// (Re, Im) h'_k, Y col 2i + c = (Re, Im) L_i, Y cols 2 KH, 2 KH + 1 = S0.
template <int KH>
struct OT {
  static constexpr int K = 2 * KH;                       // A columns
  static constexpr int N = (2 * KH + 2 + 15) / 16 * 16;  // accumulator columns per class
  static constexpr int PARTS = KH / 4;                   // builder threads per row
  static constexpr int BUILDERS = 128 * PARTS;
  static constexpr int BWARPS = BUILDERS / 32;
  static constexpr int THREADS = BUILDERS + 32;          // + the MMA issuer warp
  static constexpr uint32_t SB = (uint32_t)N * K * 4;    // one B tile (hi or lo)
  static constexpr uint32_t B0 = 0;                      // resident B: [matrix][hi, lo]
  static constexpr uint32_t MISC = NBMAT * 2 * SB;       // mbarriers, tmem address, flags
  static constexpr uint32_t WM = MISC + 128;             // per-warp offset masks (u64 x 4)
  static constexpr uint32_t LGL = WM + 32;               // float[64] log(box size)
  static constexpr uint32_t CLS = LGL + 256;             // uchar[64] offset classes
  static constexpr uint32_t TOTAL = CLS + 64;
  // tensor memory: 4 rotation-class accumulators, then OT_STAGES A stages [hi, lo]
  static constexpr uint32_t A_COL = 4 * N;
  static constexpr uint32_t TMEM_USED = A_COL + OT_STAGES * 2 * K;
  static constexpr uint32_t TMEM_COLS = TMEM_USED <= 128 ? 128 : (TMEM_USED <= 256 ? 256 : 512);
};

// Gather this thread's 4 coefficients of the row's source multipole at
// offset oi, if the row's next list-2 entry is at that offset.
template <int KH>
__device__ __forceinline__ bool ot_fetch(int oi, unsigned& ecur, int& ep, int ee,
                                         const int* __restrict__ ent,
                                         const float4* __restrict__ mp32, int ND, int d, int part,
                                         float4 (&v)[2]) {
  if ((int)(ecur >> 26) != oi) return false;
  const float4* h = mp32 + ((size_t)(ecur & 0x3FFFFFFu) * ND + d) * (KH / 2) + 2 * part;
  v[0] = h[0];
  v[1] = h[1];
  ++ep;
  ecur = ep < ee ? (unsigned)ent[ep] : 0xFFFFFFFFu;
  return true;
}

// (x, y) times i^e
__device__ __forceinline__ void rot_ie(float x, float y, int e, float& a, float& b) {
  a = (e & 1) ? -y : x;
  b = (e & 1) ? x : y;
  if (e & 2) {
    a = -a;
    b = -b;
  }
}

// MMA with A from tensor memory and B from shared memory.
__device__ __forceinline__ void umma_tf32_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b,
                                             uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
          d_tmem),
      "r"(a_tmem), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

// 8 consecutive FP32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_st8(uint32_t addr, const float* v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(addr),
      "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
      "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
      "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7]))
      : "memory");
}
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
__device__ __forceinline__ void tmem_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

struct OffsetClasses {
  unsigned char c[52];  // per offset index (ox+3)*7 + (oy+3): matrix*4 + m; 255: none
};

// One CTA per SM (persistent); a tile = 128 rows = 128/ND target boxes x ND
// densities.  tbox: box | level << 26 per target; tstart: CSR offsets into
// ent (source | offset index << 26, sorted by offset index); tmask: offsets
// present per target; btab: the resident B image; mp32: FP32 multipoles
// [box][ND][KH] (zero beyond P); lo: FP64 locals [box][P][ND].
//
// Pipeline per tile, one step per offset present in the tile: the builder
// warps (thread = row x 4 coefficients) write the A rows of step g into
// tensor-memory stage g % 4 with tcgen05.st once the MMAs of step g - 4
// have released it (empty barrier, tcgen05.commit) and arrive on the
// stage's full barrier; the issuer warp waits for it and issues the step's
// MMAs (A from tensor memory, B from shared memory).  The builders' global
// loads run two steps ahead; no CTA-wide barrier sits between the steps of
// a tile.  At the end of a tile every builder thread reads back its 4
// coefficients of the 4 class accumulators and updates the FP64 locals.
template <int KH>
__global__ void __launch_bounds__(OT<KH>::THREADS, 1)
    k_m2l_tc(const int* __restrict__ tbox, const int* __restrict__ tstart,
             const unsigned long long* __restrict__ tmask, const int* __restrict__ ent, int ntgt,
             int ndsh, int P, const float4* __restrict__ btab, OffsetClasses oc,
             const double* __restrict__ boxsize, int nlev, const float4* __restrict__ mp32,
             double2* __restrict__ lo, int* __restrict__ err) {
  using L = OT<KH>;
  constexpr int K = L::K, N = L::N;
  extern __shared__ __align__(1024) char smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r = tid & 127, part = tid >> 7;
  const int ND = 1 << ndsh, tpt = 128 >> ndsh, d = r & (ND - 1);
  uint32_t* misc = reinterpret_cast<uint32_t*>(smem + L::MISC);
  // full[OT_STAGES], empty[OT_STAGES] mbarriers, 8 bytes apart
  const uint32_t full0 = smem_u32(misc), empty0 = full0 + 8 * OT_STAGES;
  volatile uint32_t* s_taddr = misc + 4 * OT_STAGES;
  volatile int* s_fail = reinterpret_cast<volatile int*>(misc + 4 * OT_STAGES + 1);
  unsigned long long* s_wm = reinterpret_cast<unsigned long long*>(smem + L::WM);
  float* LGL = reinterpret_cast<float*>(smem + L::LGL);
  unsigned char* CLS = reinterpret_cast<unsigned char*>(smem + L::CLS);

  {
    float4* dst = reinterpret_cast<float4*>(smem + L::B0);
    constexpr int nv = (int)(NBMAT * 2 * L::SB / 16);
    for (int e = tid; e < nv; e += L::THREADS) dst[e] = btab[e];
  }
  for (int e = tid; e < 64; e += L::THREADS) {
    LGL[e] = e < nlev ? (float)log(boxsize[e]) : 0.f;
    CLS[e] = e < 49 ? oc.c[e] : (unsigned char)255;
  }
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
  const long ntiles = (ntgt + tpt - 1) / tpt;
  const bool builder = warp < L::BWARPS;
  uint32_t g = 0;  // offset steps of this CTA so far; stage g % OT_STAGES
  int zmask = 0;   // bit s: this thread's columns of stage s hold zeros

  for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long ti = tile * tpt + (r >> ndsh);
    const bool valid = builder && ti < ntgt;
    int ep = 0, ee = 0;
    unsigned long long msk = 0;
    if (valid) {
      ep = tstart[ti];
      ee = tstart[ti + 1];
      msk = tmask[ti];
    }
    {
      unsigned a = __reduce_or_sync(~0u, (unsigned)msk);
      unsigned b = __reduce_or_sync(~0u, (unsigned)(msk >> 32));
      if (lane == 0 && warp < 4) s_wm[warp] = ((unsigned long long)b << 32) | a;
    }
    __syncthreads();
    if (*s_fail) break;
    const unsigned long long mask = s_wm[0] | s_wm[1] | s_wm[2] | s_wm[3];
    const uint32_t g0 = g, nsteps = (uint32_t)__popcll(mask);

    if (builder) {
      unsigned ecur = ep < ee ? (unsigned)ent[ep] : 0xFFFFFFFFu;
      unsigned long long fm = mask;  // offsets not fetched yet
      float4 va[2], vb[2], vc[2];
      int oa = -1, ob = -1;
      bool ha = false, hb = false;
      if (fm) {
        oa = __ffsll((long long)fm) - 1;
        fm &= fm - 1;
        ha = ot_fetch<KH>(oa, ecur, ep, ee, ent, mp32, ND, d, part, va);
      }
      if (fm) {
        ob = __ffsll((long long)fm) - 1;
        fm &= fm - 1;
        hb = ot_fetch<KH>(ob, ecur, ep, ee, ent, mp32, ND, d, part, vb);
      }
      int pend = -1;  // stage whose stores are in flight (arrival deferred by one step)
      while (oa >= 0) {
        bool hc = false;
        int ocn = -1;
        if (fm) {
          ocn = __ffsll((long long)fm) - 1;
          fm &= fm - 1;
          hc = ot_fetch<KH>(ocn, ecur, ep, ee, ent, mp32, ND, d, part, vc);
        }
        const int s = (int)(g % OT_STAGES);
        if (g >= OT_STAGES && !*s_fail) {
          if (!mbar_wait_backoff(empty0 + 8 * s, (g / OT_STAGES - 1) & 1)) *s_fail = 1;
          tc_fence_after();
        }
        // coefficient k = 4 part + j, so k = j (mod 4): input phase i^(-m j)
        float hi[8], lw[8];
        {
          const int m = CLS[oa] & 3;
          const float x[4] = {va[0].x, va[0].z, va[1].x, va[1].z};
          const float y[4] = {va[0].y, va[0].w, va[1].y, va[1].w};
#pragma unroll
          for (int j = 0; j < 4; j++) {
            float a = 0.f, b = 0.f;
            if (ha) rot_ie(x[j], y[j], (-(m * j)) & 3, a, b);
            hi[2 * j] = tf32_rna(a);
            hi[2 * j + 1] = tf32_rna(b);
            lw[2 * j] = a - hi[2 * j];
            lw[2 * j + 1] = b - hi[2 * j + 1];
          }
        }
        // the previous step's rows are in tensor memory: publish them
        if (pend >= 0) {
          tmem_wait_st();
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(full0 + 8 * pend);
        }
        // tcgen05.st is warp-collective: the warp writes when any of its rows
        // changes (new data, or zeros over data)
        const bool need = ha || !((zmask >> s) & 1);
        if (__any_sync(~0u, need)) {
          const uint32_t acol = lane_base + L::A_COL + (uint32_t)(s * 2 * K) + 8 * part;
          tmem_st8(acol, hi);
          tmem_st8(acol + K, lw);
        }
        zmask = ha ? (zmask & ~(1 << s)) : (zmask | (1 << s));
        pend = s;
        ++g;
        oa = ob;
        ha = hb;
        ob = ocn;
        hb = hc;
        va[0] = vb[0];
        va[1] = vb[1];
        vb[0] = vc[0];
        vb[1] = vc[1];
      }
      if (pend >= 0) {
        tmem_wait_st();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(full0 + 8 * pend);
      }
    } else if (lane == 0) {
      // MMA issuer.  After the blocking wait for the next stage it also takes
      // the following stages that are already full, so that one tcgen05 fence
      // covers several steps (the fence costs a few hundred clocks), and it
      // reads the next step's class ahead of time.
      const uint32_t idesc = idesc_tf32(TC_ROWS, N);
      unsigned touched = 0;
      bool fail = *s_fail != 0;
      unsigned long long mm = mask;
      int cl_next = mm ? CLS[__ffsll((long long)mm) - 1] : 255;
      uint32_t left = nsteps;
      while (left > 0) {
        if (!fail && !mbar_wait(full0 + 8 * (g % OT_STAGES), (g / OT_STAGES) & 1)) fail = true;
        uint32_t ready = 1;
        while (!fail && ready < left && ready < OT_STAGES) {
          const uint32_t gn = g + ready;
          if (!mbar_test(full0 + 8 * (gn % OT_STAGES), (gn / OT_STAGES) & 1)) break;
          ++ready;
        }
        tc_fence_after();
        for (uint32_t q = 0; q < ready; q++) {
          mm &= mm - 1;
          const int cl = cl_next;
          cl_next = mm ? CLS[__ffsll((long long)mm) - 1] : 255;
          const int s = (int)(g % OT_STAGES);
          if (cl == 255) fail = true;  // not an interaction offset: its MMA is not issued
          if (!fail) {
            const int m = cl & 3;
            const uint32_t a_hi = taddr + L::A_COL + (uint32_t)(s * 2 * K), a_lo = a_hi + K;
            // descriptors of the matrix's hi and lo tiles; a K step of 8 columns
            // advances the start address by 256 bytes (16 in descriptor units)
            const uint64_t bh = umma_desc(sbase + L::B0 + (uint32_t)(cl >> 2) * 2 * L::SB, 128,
                                          (uint32_t)K * 32);
            const uint64_t bl = bh + (L::SB >> 4);
            const uint32_t dt = taddr + (uint32_t)(m * N);
            const uint32_t acc0 = ((touched >> m) & 1u) ? 1u : 0u;
#pragma unroll
            for (int ks = 0; ks < K / 8; ks++) {
              umma_tf32_ts(dt, a_hi + 8 * ks, bh + 16 * ks, idesc, ks == 0 ? acc0 : 1u);
              umma_tf32_ts(dt, a_hi + 8 * ks, bl + 16 * ks, idesc, 1u);
              umma_tf32_ts(dt, a_lo + 8 * ks, bh + 16 * ks, idesc, 1u);
            }
            touched |= 1u << m;
          }
          // the commit also releases the stage when nothing was issued
          umma_commit(empty0 + 8 * s);
          ++g;
        }
        left -= ready;
      }
      if (fail) *s_fail = 1;
    }
    g = g0 + nsteps;
    // rotation classes present in the tile (the same on every thread)
    unsigned touched = 0;
    for (unsigned long long mm = mask; mm; mm &= mm - 1)
      touched |= 1u << (CLS[__ffsll((long long)mm) - 1] & 3);
    if (nsteps > 0 && builder) {
      // epilogue: the last commit of the tile covers all of its MMAs
      const uint32_t gl = g - 1;
      if (!mbar_wait(empty0 + 8 * (gl % OT_STAGES), (gl / OT_STAGES) & 1)) *s_fail = 1;
      tc_fence_after();
      float acc[8], s0[2] = {0.f, 0.f};
#pragma unroll
      for (int i = 0; i < 8; i++) acc[i] = 0.f;
      for (int m = 0; m < 4; m++) {
        if (!((touched >> m) & 1u)) continue;
        float y[8];
        tmem_ld8(lane_base + (uint32_t)(m * N + 8 * part), y);
        tmem_wait_ld();
#pragma unroll
        for (int q = 0; q < 4; q++) {
          // coefficient i = 4 part + q: output phase i^(-m i) = i^(-m q)
          float a, b;
          rot_ie(y[2 * q], y[2 * q + 1], (-(m * q)) & 3, a, b);
          acc[2 * q] += a;
          acc[2 * q + 1] += b;
        }
        if (part == 0) {
          tmem_ld8(lane_base + (uint32_t)(m * N + 2 * KH), y);
          tmem_wait_ld();
          s0[0] += y[0];
          s0[1] += y[1];
        }
      }
      if (valid && !*s_fail) {
        const unsigned tb = (unsigned)tbox[ti];
        if (part == 0) {
          const float lg = LGL[tb >> 26];
          acc[0] += lg * s0[0];
          acc[1] += lg * s0[1];
        }
        double2* out = lo + ((size_t)(tb & 0x3FFFFFFu) * P + 4 * part) * ND + d;
#pragma unroll
        for (int q = 0; q < 4; q++) {
          if (4 * part + q < P) {
            double2 v = out[(size_t)q * ND];
            v.x += (double)acc[2 * q];
            v.y += (double)acc[2 * q + 1];
            out[(size_t)q * ND] = v;
          }
        }
      }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  if (*s_fail && g > 0) {
    // the tensor cores may still be working: one more bounded wait for the
    // last commit before the tensor memory is released
    const uint32_t gl = g - 1;
    mbar_wait(empty0 + 8 * (gl % OT_STAGES), (gl / OT_STAGES) & 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(taddr, L::TMEM_COLS);
  if (tid == 0 && *s_fail) atomicExch(err, 1);
}

// B image of the 14 resident operators (7 base offsets, each as is and
// conjugated): [matrix][hi, lo][N x K canonical layout], interleaved columns.
__global__ void k_m2l_btab(int KH, int N, int P, const double* __restrict__ binom,
                           float* __restrict__ out) {
  const int K = 2 * KH;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= NBMAT * N * K) return;
  const int mat = e / (N * K), rem = e % (N * K), n = rem / K, kc = rem % K;
  const int b = mat >> 1;
  const bool conj = mat & 1;
  const double ox = base_ox(b), oy = base_oy(b), den = ox * ox + oy * oy;
  const double ur = ox / den, ui = -oy / den;  // u = 1/o
  double v = 0.0;
  if (n < 2 * KH) {
    const int i = n >> 1, k = kc >> 1;
    const bool im_out = n & 1, im_in = kc & 1;
    if (i < P && k < P) {
      double tr, tim;
      if (i == 0 && k == 0) {
        tr = 0.5 * log(den);
        tim = 0.0;
      } else {
        double gik;
        if (i == 0)
          gik = 1.0;
        else if (k == 0)
          gik = -1.0 / i;
        else
          gik = binom[(size_t)(i + k - 1) * BINOM_N + (k - 1)];
        double pr = 1.0, pi = 0.0;  // u^(i+k)
        for (int q = 0; q < i + k; q++) {
          const double t = pr * ur - pi * ui;
          pi = pr * ui + pi * ur;
          pr = t;
        }
        const double sg = (k & 1) ? -gik : gik;  // u^i (-u)^k
        tr = sg * pr;
        tim = sg * pi;
      }
      if (conj) tim = -tim;
      v = (im_out == im_in) ? tr : (im_out ? tim : -tim);
    }
  } else if ((n == 2 * KH && kc == 0) || (n == 2 * KH + 1 && kc == 1)) {
    v = 1.0;
  }
  const float hi = tf32_rna((float)v), lw = (float)(v - (double)hi);
  const uint32_t o = tile_off(n, kc, K) / 4;
  out[(size_t)mat * 2 * N * K + o] = hi;
  out[(size_t)mat * 2 * N * K + (size_t)N * K + o] = lw;
}

// FP32 copy of one density chunk's multipoles, [box][ND][KH] (zero beyond P).
__global__ void k_mp_to_f32(const double2* __restrict__ mp, long nbox, int P, int ND, int KH,
                            float2* __restrict__ out) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= nbox * ND * KH) return;
  const int k = (int)(e % KH);
  const long bd = e / KH;
  const int d = (int)(bd % ND);
  const long box = bd / ND;
  float2 v = make_float2(0.f, 0.f);
  if (k < P) {
    const double2 x = mp[((size_t)box * P + k) * ND + d];
    v = make_float2((float)x.x, (float)x.y);
  }
  out[e] = v;
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

__global__ void k_m2l_flag(TV t, int first, int n, int* __restrict__ flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int b = first + i;
  flag[i] = (t.has_eval_pts(b) && t.nl2[b] > 0) ? 1 : 0;
}

// Compact the targets with their child position (parity of the box's grid
// coordinates at its level), which fixes the set of list-2 offsets a box
// can have: targets grouped by it make tiles of at most 27 offsets.
__global__ void k_m2l_compact(TV t, int first, int n, const int* __restrict__ flag,
                              const int* __restrict__ tix, int* __restrict__ key,
                              int* __restrict__ box) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !flag[i]) return;
  const int b = first + i;
  const double bs = t.boxsize[t.level[b]];
  const double2 c = t.center[b], c0 = t.center[0];
  const double h0 = 0.5 * t.boxsize[0];
  const long ix = __double2ll_rn((c.x - c0.x + h0) / bs - 0.5);
  const long iy = __double2ll_rn((c.y - c0.y + h0) / bs - 0.5);
  key[tix[i]] = (int)((ix & 1) | ((iy & 1) << 1));
  box[tix[i]] = b;
}

__global__ void k_m2l_count(TV t, const int* __restrict__ box, int ntgt, int* __restrict__ cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ntgt) cnt[i] = t.nl2[box[i]];
}

// Target boxes and their list-2 entries sorted by offset index.
__global__ void k_m2l_fill(TV t, const int* __restrict__ box, int ntgt, const int* __restrict__ cnt,
                           const int* __restrict__ offs, int* __restrict__ tbox,
                           int* __restrict__ tstart, unsigned long long* __restrict__ tmask,
                           int* __restrict__ ent) {
  const int ti = blockIdx.x * blockDim.x + threadIdx.x;
  if (ti >= ntgt) return;
  const int b = box[ti], n2 = cnt[ti];
  const double2 cb = t.center[b];
  const double rinv = 1.0 / t.boxsize[t.level[b]];
  unsigned key[MNLIST2];
  unsigned long long mask = 0;
  for (int e = 0; e < n2; e++) {
    const int jb = t.l2[(size_t)MNLIST2 * b + e];
    const double2 cj = t.center[jb];
    const int ox = __double2int_rn((cj.x - cb.x) * rinv), oy = __double2int_rn((cj.y - cb.y) * rinv);
    const unsigned oi = (unsigned)((ox + 3) * 7 + (oy + 3));
    unsigned k = (unsigned)jb | (oi << 26);
    int q = e;
    while (q > 0 && key[q - 1] > k) {
      key[q] = key[q - 1];
      q--;
    }
    key[q] = k;
    mask |= 1ull << oi;
  }
  const int o = offs[ti];
  for (int e = 0; e < n2; e++) ent[o + e] = (int)key[e];
  tbox[ti] = (int)((unsigned)b | ((unsigned)t.level[b] << 26));
  tstart[ti] = o;
  tmask[ti] = mask;
}

__global__ void k_set_int(int* p, int v) { *p = v; }

// Offset-steps of all tiles of 128/ND targets (the issued tensor-core work).
__global__ void k_m2l_steps(const unsigned long long* __restrict__ tmask, long ntgt, int tpt,
                            unsigned long long* __restrict__ out) {
  const long tile = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (tile * tpt >= ntgt) return;
  unsigned long long m = 0;
  for (long q = tile * tpt; q < min(ntgt, (tile + 1) * tpt); q++) m |= tmask[q];
  atomicAdd(out, (unsigned long long)__popcll(m));
}

// Offset o = i^m b or i^m conj(b) for a base offset b: resident matrix
// 2 b (+1 for the conjugate) and rotation class m.
OffsetClasses offset_classes() {
  OffsetClasses oc;
  for (auto& c : oc.c) c = 255;
  for (int oi = 0; oi < 49; oi++) {
    const int ox = oi / 7 - 3, oy = oi % 7 - 3;
    if (std::max(std::abs(ox), std::abs(oy)) < 2) continue;
    bool found = false;
    for (int b = 0; b < NBASE && !found; b++)
      for (int c = 0; c < 2 && !found; c++) {
        int x = base_ox(b), y = c ? -base_oy(b) : base_oy(b);
        for (int m = 0; m < 4 && !found; m++) {
          if (x == ox && y == oy) {
            oc.c[oi] = (unsigned char)((2 * b + c) * 4 + m);
            found = true;
          }
          const int t = x;  // times i
          x = -y;
          y = t;
        }
      }
  }
  return oc;
}

int m2l_kh(int P) { return (P + 3) / 4 * 4; }

}  // namespace

bool m2l_tc_supported(int P) { return P >= 2 && P <= 20; }

void m2l_tc_build(M2LPairs& L, const TV& t, int first, int n, int nboxes, int P, int chunk,
                  cudaStream_t st) {
  L.ntgt = L.npairs = 0;
  L.P = P;
  L.usable = nboxes < (1 << 26) && m2l_tc_supported(P);
  if (!L.usable || n <= 0) return;
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
  int* h = pinned_ints(2);
  B2_CHECK(cudaMemcpyAsync(h, tix.p + (n - 1), sizeof(int), cudaMemcpyDeviceToHost, st));
  B2_CHECK(cudaMemcpyAsync(h + 1, flag.p + (n - 1), sizeof(int), cudaMemcpyDeviceToHost, st));
  B2_CHECK(cudaStreamSynchronize(st));
  const int ntgt = h[0] + h[1];
  if (ntgt == 0) return;
  // targets grouped by child position (stable: box order inside a group)
  DBuf<int> key(st), box(st), skey(st), sbox(st), cnt(st), offs(st);
  key.alloc(ntgt, st);
  box.alloc(ntgt, st);
  skey.alloc(ntgt, st);
  sbox.alloc(ntgt, st);
  k_m2l_compact<<<ceil_div(n, 256), 256, 0, st>>>(t, first, n, flag.p, tix.p, key.p, box.p);
  B2_LAUNCH_CHECK();
  size_t tb2 = 0;
  B2_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, tb2, key.p, skey.p, box.p, sbox.p, ntgt, 0, 2,
                                           st));
  DBuf<char> tmp2(st);
  tmp2.alloc(tb2, st);
  B2_CHECK(cub::DeviceRadixSort::SortPairs(tmp2.p, tb2, key.p, skey.p, box.p, sbox.p, ntgt, 0, 2,
                                           st));
  cnt.alloc(ntgt, st);
  offs.alloc(ntgt, st);
  k_m2l_count<<<ceil_div(ntgt, 256), 256, 0, st>>>(t, sbox.p, ntgt, cnt.p);
  B2_LAUNCH_CHECK();
  size_t tb3 = 0;
  B2_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, tb3, cnt.p, offs.p, ntgt, st));
  DBuf<char> tmp3(st);
  tmp3.alloc(tb3, st);
  B2_CHECK(cub::DeviceScan::ExclusiveSum(tmp3.p, tb3, cnt.p, offs.p, ntgt, st));
  B2_CHECK(cudaMemcpyAsync(h, offs.p + (ntgt - 1), sizeof(int), cudaMemcpyDeviceToHost, st));
  B2_CHECK(cudaMemcpyAsync(h + 1, cnt.p + (ntgt - 1), sizeof(int), cudaMemcpyDeviceToHost, st));
  B2_CHECK(cudaStreamSynchronize(st));
  L.ntgt = ntgt;
  L.npairs = (long)h[0] + h[1];
  L.tbox.alloc(L.ntgt, st);
  L.tstart.alloc(L.ntgt + 1, st);
  L.tmask.alloc(L.ntgt, st);
  L.ent.alloc(std::max<long>(L.npairs, 1), st);
  k_m2l_fill<<<ceil_div(ntgt, 128), 128, 0, st>>>(t, sbox.p, ntgt, cnt.p, offs.p, L.tbox.p,
                                                  L.tstart.p, L.tmask.p, L.ent.p);
  B2_LAUNCH_CHECK();
  k_set_int<<<1, 1, 0, st>>>(L.tstart.p + L.ntgt, (int)L.npairs);
  B2_LAUNCH_CHECK();
  const int KH = m2l_kh(P), K = 2 * KH, N = (2 * KH + 2 + 15) / 16 * 16;
  L.btab.alloc((size_t)NBMAT * 2 * N * K, st);
  k_m2l_btab<<<ceil_div(NBMAT * N * K, 256), 256, 0, st>>>(KH, N, P, device_binomials(), L.btab.p);
  B2_LAUNCH_CHECK();
  L.steps.alloc(1, st);
  L.steps.zero(1);
  const int tpt = 128 / chunk;
  k_m2l_steps<<<ceil_div(ceil_div(L.ntgt, tpt), 128), 128, 0, st>>>(L.tmask.p, L.ntgt, tpt,
                                                                    L.steps.p);
  B2_LAUNCH_CHECK();
  // the temporaries above are freed (stream-ordered) when this returns
}

long m2l_tc_scratch(const M2LPairs& L, int nboxes, int ND) {
  return (long)nboxes * ND * m2l_kh(L.P);
}

int m2l_tc_run(int ND, const M2LPairs& L, const double2* mp, float2* mp32, long nmp32, int nboxes,
               double2* lo, const double* boxsize, int nlev, int* err_dev, cudaStream_t st) {
  if (L.npairs == 0) return IER_OK;
  const int P = L.P;
  if (nlev > 64 || !m2l_tc_supported(P) || !(ND == 1 || ND == 2 || ND == 4 || ND == 8))
    return IER_BADARG;
  if (nmp32 < m2l_tc_scratch(L, nboxes, ND)) return IER_BADARG;
  const int KH = m2l_kh(P);
  const int ndsh = ND == 8 ? 3 : (ND == 4 ? 2 : (ND == 2 ? 1 : 0));
  int dev = 0, nsm = 148;
  B2_CHECK(cudaGetDevice(&dev));
  B2_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const long nconv = (long)nboxes * ND * KH;
  k_mp_to_f32<<<ceil_div(nconv, 256), 256, 0, st>>>(mp, nboxes, P, ND, KH, mp32);
  B2_LAUNCH_CHECK();
  const OffsetClasses oc = offset_classes();
  const long ntiles = (L.ntgt + (128 >> ndsh) - 1) / (128 >> ndsh);
  auto launch = [&](auto kern, uint32_t total, uint32_t tmem_cols, int threads) {
    // CTAs that can share an SM's 512 tensor-memory columns; the shared
    // memory request keeps more from being resident (an allocation would wait)
    const int per_sm = 512 / (int)tmem_cols;
    const size_t sm = std::max<size_t>(total, (size_t)(233472 / (per_sm + 1)) + 1024);
    set_smem_attr(kern, sm);
    const int grid = (int)std::min<long>(ntiles, (long)nsm * per_sm);
    kern<<<grid, threads, sm, st>>>(L.tbox.p, L.tstart.p, L.tmask.p, L.ent.p, (int)L.ntgt, ndsh,
                                    P, reinterpret_cast<const float4*>(L.btab.p), oc, boxsize,
                                    nlev, reinterpret_cast<const float4*>(mp32), lo, err_dev);
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
