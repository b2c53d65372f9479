// M2L of the mixed-precision Laplace FMM on the 5th-generation tensor cores.
//
// The translation of laprouts2d.f:1130-1244 between boxes of one level is,
// on scaled expansions and with the integer offset o = (c_src - c_tgt) / bs
// and u = 1/o,
//     t_j = h_j (-u)^j,   y = G t,   L_i += u^i y_i,   L_0 += t_0 log|z0|,
// with the real matrix G_0j = 1 (j > 0), G_i0 = -1/i, G_ij = C(i+j-1, j-1)
// shared by every pair.  All pairs of the FMM form one GEMM
//     Y[rows, :] = T[rows, :] G^T,   rows = (pair, density),
// which runs here as 128-row tiles: the CTA's threads build the T tile (one
// row each: the source multipole times the powers of -u, split into TF32
// hi + lo) directly in the UMMA canonical K-major layout in shared memory,
// one thread issues tcgen05.mma (kind::tf32, M = 128, N = 16/32, K = 8 per
// instruction; the three products hi*hi + hi*lo + lo*hi give FP32-level
// accuracy) into a tensor-memory accumulator, and after the commit barrier
// every thread reads its row back with tcgen05.ld, applies u^i and the log
// term, and the rows of each target box are summed through shared memory
// and added to its FP64 local expansion.
//
// Shared-memory operand layout (no swizzle, K-major): element (r, k) of a
// tile with K columns sits at byte (r/8)*SBO + (k/4)*128 + (r%8)*16 + (k%4)*4,
// SBO = 32 K: 8x16-byte core matrices, K-adjacent core matrices 128 bytes
// apart (leading byte offset), 8-row groups SBO apart (stride byte offset).
//
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
constexpr long TC_WAIT_LIMIT = 1L << 22;  // polls of the commit barrier (~0.5 s)

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

__device__ __forceinline__ void mbar_init(uint32_t mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for the given phase parity of the barrier.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (long it = 0; it < TC_WAIT_LIMIT; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (it > 64) __nanosleep(64);
  }
  return false;
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

struct TcSmem {
  // byte offsets inside the dynamic shared memory
  uint32_t a, b, u, lg, lgl, tgt, wsum, gstart, misc;
  uint32_t total;
};

__host__ __device__ inline TcSmem tc_layout(int P, int K, int N) {
  TcSmem s;
  const uint32_t SA = 128u * K * 4, SB = (uint32_t)N * K * 4;
  s.a = 0;                       // A: re_hi, re_lo, im_hi, im_lo (reused for row results)
  s.b = 4 * SA;                  // B: hi, lo
  s.u = s.b + 2 * SB;            // float2 [49][P]
  s.lg = s.u + 49u * P * 8;      // float [49]
  s.lgl = s.lg + 49 * 4;         // float [64] log(boxsize) per level
  s.tgt = (s.lgl + 64 * 4 + 15) & ~15u;  // int [128] target of each pair of the tile
  s.wsum = s.tgt + 128 * 4;      // int [4]
  s.gstart = s.wsum + 16;        // int [132]
  s.misc = (s.gstart + 132 * 4 + 15) & ~15u;  // mbarrier (8), taddr (4), fail (4), ngroups (4)
  s.total = s.misc + 32;
  return s;
}

// G^T as the N x K B operand (row i, column j = G_ij), split into hi / lo.
__device__ void build_g(char* smem, const TcSmem& L, int P, int K, int N,
                        const double* __restrict__ binom) {
  char* bhi = smem + L.b;
  char* blo = bhi + N * K * 4;
  for (int e = threadIdx.x; e < N * (K / 4); e += blockDim.x) {
    int i = e / (K / 4), j0 = (e % (K / 4)) * 4;
    float g[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      int j = j0 + q;
      float v = 0.f;
      if (i < P && j < P) {
        if (i == 0)
          v = (j == 0) ? 0.f : 1.f;
        else if (j == 0)
          v = -1.f / i;
        else
          v = (float)binom[(size_t)(i + j - 1) * BINOM_N + (j - 1)];
      }
      g[q] = v;
    }
    store_split4(bhi, blo, i, j0, K, g[0], g[1], g[2], g[3]);
  }
}

// FP32 copy of the multipoles of one density chunk ([box][P][ND] float2).
__global__ void k_mp_to_f32(const double2* __restrict__ mp, long n, float2* __restrict__ out) {
  long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k < n) out[k] = make_float2((float)mp[k].x, (float)mp[k].y);
}

// One tile = 128 rows = TP = 128 / ND pairs x ND densities; thread = row.
// Software pipeline per CTA: the pair metadata and source multipoles of the
// next tile are loaded into registers right after the current tile's MMAs
// are issued, so their latency hides behind the tensor-core work, the
// tensor-memory read-back and the reduction of the current tile.
template <int ND, int K>
__global__ void __launch_bounds__(128, 3)
    k_m2l_tc(const int2* __restrict__ pairs, long npairs, int P, int N,
             const double* __restrict__ binom, const float2* __restrict__ utab_g,
             const float* __restrict__ lgtab_g, const double* __restrict__ boxsize, int nlev,
             const float2* __restrict__ mp32, double2* __restrict__ lo, int* __restrict__ err) {
  extern __shared__ __align__(1024) char smem[];
  const TcSmem L = tc_layout(P, K, N);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr uint32_t SA = 128u * K * 4;
  char* A = smem + L.a;
  float2* U = reinterpret_cast<float2*>(smem + L.u);
  float* LG = reinterpret_cast<float*>(smem + L.lg);
  float* LGL = reinterpret_cast<float*>(smem + L.lgl);
  int* s_tgt = reinterpret_cast<int*>(smem + L.tgt);
  int* s_wsum = reinterpret_cast<int*>(smem + L.wsum);
  int* s_gstart = reinterpret_cast<int*>(smem + L.gstart);
  uint32_t* misc = reinterpret_cast<uint32_t*>(smem + L.misc);
  const uint32_t mbar = smem_u32(misc);  // misc[0..1]
  volatile uint32_t* s_taddr = misc + 2;
  volatile int* s_fail = reinterpret_cast<volatile int*>(misc + 4);

  build_g(smem, L, P, K, N, binom);
  for (int e = tid; e < 49 * P; e += blockDim.x) U[e] = utab_g[e];
  for (int e = tid; e < 49; e += blockDim.x) LG[e] = lgtab_g[e];
  for (int e = tid; e < 64; e += blockDim.x) LGL[e] = e < nlev ? (float)log(boxsize[e]) : 0.f;
  if (tid == 0) {
    mbar_init(mbar);
    *s_fail = 0;
  }
  __syncwarp();
  if (warp == 0) tmem_alloc(smem_u32((const void*)s_taddr), TC_TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t taddr = *s_taddr;
  const uint32_t idesc = idesc_tf32(TC_ROWS, N);
  const uint32_t a_base = smem_u32(A), b_base = smem_u32(smem + L.b);
  constexpr int TP = TC_ROWS / ND;  // pairs per tile
  const long ntiles = (npairs + TP - 1) / TP;
  const int row = tid, pl = row / ND, d = row % ND;
  uint32_t parity = 0;
  float* R = reinterpret_cast<float*>(A);  // row results [128][2P], after the MMA

  // registers of the tile being prepared: pair, previous pair's target,
  // source multipole
  int2 pr = make_int2(-1, 0);
  int prev_tgt = -1;
  float2 hv[K];
  auto fetch = [&](long tile) {
    long p = tile * TP + pl;
    pr = make_int2(-1, 0);
    prev_tgt = -1;
    if (tile < ntiles && p < npairs) {
      pr = pairs[p];
      if (pl > 0) prev_tgt = pairs[p - 1].x;
      int src = pr.y & 0x3FFFFFF;
      const float2* h = mp32 + (size_t)src * P * ND + d;
#pragma unroll
      for (int j = 0; j < K; j++) hv[j] = j < P ? h[(size_t)j * ND] : make_float2(0.f, 0.f);
    }
  };
  fetch(blockIdx.x);

  for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const bool valid = pr.x >= 0;
    const int tgt = valid ? (pr.x & 0x3FFFFFF) : -1;
    const int lev = valid ? (int)((unsigned)pr.x >> 26) : 0;
    const int oi = valid ? (int)((unsigned)pr.y >> 26) : 24;
    const float lge = LGL[lev] + LG[oi];
    // group starts: a pair opens a group when its target differs from the
    // previous pair's (block-wide scan of the flags)
    int flag = 0;
    if (valid && d == 0) flag = (pl == 0) || ((prev_tgt & 0x3FFFFFF) != tgt);
    int incl = flag;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int v = __shfl_up_sync(~0u, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) s_wsum[warp] = incl;
    if (d == 0) s_tgt[pl] = tgt;
    // T row: t_j = h_j (-u)^j, split into TF32 hi + lo
    float2 t0 = make_float2(0.f, 0.f);
#pragma unroll
    for (int j0 = 0; j0 < K; j0 += 4) {
      float re[4], im[4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        int j = j0 + q;
        float2 v = make_float2(0.f, 0.f);
        if (valid && j < P) {
          float2 s = U[oi * P + j];
          if (j & 1) s = make_float2(-s.x, -s.y);
          v = make_float2(hv[j].x * s.x - hv[j].y * s.y, hv[j].x * s.y + hv[j].y * s.x);
        }
        if (j == 0) t0 = v;
        re[q] = v.x;
        im[q] = v.y;
      }
      store_split4(A, A + SA, row, j0, K, re[0], re[1], re[2], re[3]);
      store_split4(A + 2 * SA, A + 3 * SA, row, j0, K, im[0], im[1], im[2], im[3]);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      issue_split_mma(taddr, a_base, a_base + SA, b_base, b_base + N * K * 4, K, idesc);
      issue_split_mma(taddr + (uint32_t)N, a_base + 2 * SA, a_base + 3 * SA, b_base,
                      b_base + N * K * 4, K, idesc);
      umma_commit(mbar);
    }
    // group index of the flagged pairs
    {
      int pre = 0;
      for (int w = 0; w < warp; w++) pre += s_wsum[w];
      if (flag) s_gstart[pre + incl - 1] = pl;
      if (tid == blockDim.x - 1) misc[5] = pre + incl;  // number of groups
    }
    const long tile_first = tile * TP;
    const int tile_pairs = (int)min((long)TP, npairs - tile_first);
    // the next tile's loads overlap the tensor-core work
    fetch(tile + gridDim.x);
    bool ok = mbar_wait(mbar, parity);
    parity ^= 1u;
    if (!ok) *s_fail = 1;
    tc_fence_after();
    // L_i contribution u^i y_i (+ t_0 log|z0| at i = 0), staged as rows in the
    // A tiles, which the completed MMAs no longer read
    const uint32_t lane_addr = taddr + ((uint32_t)(warp * 32) << 16);
    float* Rr = R + (size_t)row * 2 * P;
#pragma unroll
    for (int c0 = 0; c0 < 32; c0 += 16) {
      if (c0 >= N) break;
      float yr[16], yi[16];
      tmem_ld16(lane_addr + c0, yr);
      tmem_ld16(lane_addr + (uint32_t)N + c0, yi);
      tmem_wait_ld();
#pragma unroll
      for (int q = 0; q < 16; q++) {
        int i = c0 + q;
        if (i >= P) break;
        float zr, zi;
        if (i == 0) {
          zr = yr[0] + t0.x * lge;
          zi = yi[0] + t0.y * lge;
        } else {
          float2 ui = U[oi * P + i];
          zr = yr[q] * ui.x - yi[q] * ui.y;
          zi = yr[q] * ui.y + yi[q] * ui.x;
        }
        Rr[2 * i] = valid ? zr : 0.f;
        Rr[2 * i + 1] = valid ? zi : 0.f;
      }
    }
    tc_fence_before();
    __syncthreads();
    // sum the rows of every target box into its local expansion; target
    // boxes at the tile ends may also receive rows from the neighbouring
    // tiles, so every update is an atomic add (its result is not used, so it
    // does not wait for the memory system)
    const int ngroups = (int)misc[5];
    const int comps = 2 * P * ND;
    for (int w = tid; w < ngroups * comps; w += blockDim.x) {
      int g = w / comps, c = w % comps;
      int dd = c % ND, ic = c / ND, i = ic >> 1, part = ic & 1;
      int g0 = s_gstart[g], g1 = (g + 1 < ngroups) ? s_gstart[g + 1] : tile_pairs;
      float sum = 0.f;
      for (int q = g0; q < g1; q++) sum += R[(size_t)(q * ND + dd) * 2 * P + 2 * i + part];
      int tb = s_tgt[g0];
      atomicAdd(reinterpret_cast<double*>(&lo[((size_t)tb * P + i) * ND + dd]) + part,
                (double)sum);
    }
    __syncthreads();
    if (*s_fail) {
      // the tensor cores may still be working on this tile: give them one more
      // bounded wait before the tensor memory is released
      mbar_wait(mbar, parity ^ 1u);
      break;
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(taddr, TC_TMEM_COLS);
  if (tid == 0 && *s_fail) atomicExch(err, 1);
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

__global__ void k_pair_count(TV t, int first, int n, int* __restrict__ cnt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b = first + i;
  cnt[i] = t.has_eval_pts(b) ? t.nl2[b] : 0;
}

__global__ void k_pair_fill(TV t, int first, int n, const int* __restrict__ offs,
                            int2* __restrict__ pairs) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b = first + i;
  if (!t.has_eval_pts(b)) return;
  int n2 = t.nl2[b];
  double2 cb = t.center[b];
  double rinv = 1.0 / t.boxsize[t.level[b]];
  long o = offs[i];
  for (int e = 0; e < n2; e++) {
    int jb = t.l2[(size_t)MNLIST2 * b + e];
    double2 cj = t.center[jb];
    int ox = __double2int_rn((cj.x - cb.x) * rinv), oy = __double2int_rn((cj.y - cb.y) * rinv);
    int oi = (ox + 3) * 7 + (oy + 3);
    pairs[o + e] = make_int2((int)((unsigned)b | ((unsigned)t.level[b] << 26)),
                             (int)((unsigned)jb | ((unsigned)oi << 26)));
  }
}

}  // namespace

bool m2l_tc_supported(int P) { return P >= 2 && P <= 32; }

void m2l_tc_build_pairs(M2LPairs& L, const TV& t, int first, int n, int nboxes, cudaStream_t st) {
  L.npairs = 0;
  L.usable = nboxes < (1 << 26);
  if (!L.usable || n <= 0) return;
  DBuf<int> cnt(st), offs(st);
  cnt.alloc(n, st);
  offs.alloc(n, st);
  k_pair_count<<<ceil_div(n, 256), 256, 0, st>>>(t, first, n, cnt.p);
  B2_LAUNCH_CHECK();
  size_t tb = 0;
  B2_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.p, offs.p, n, st));
  DBuf<char> tmp(st);
  tmp.alloc(tb, st);
  B2_CHECK(cub::DeviceScan::ExclusiveSum(tmp.p, tb, cnt.p, offs.p, n, st));
  int* h = pinned_ints(2);
  B2_CHECK(cudaMemcpyAsync(h, offs.p + (n - 1), sizeof(int), cudaMemcpyDeviceToHost, st));
  B2_CHECK(cudaMemcpyAsync(h + 1, cnt.p + (n - 1), sizeof(int), cudaMemcpyDeviceToHost, st));
  B2_CHECK(cudaStreamSynchronize(st));
  L.npairs = (long)h[0] + h[1];
  if (L.npairs == 0) return;
  L.pairs.alloc(L.npairs, st);
  k_pair_fill<<<ceil_div(n, 256), 256, 0, st>>>(t, first, n, offs.p, L.pairs.p);
  B2_LAUNCH_CHECK();
}

int m2l_tc_run(int ND, const TV& t, const M2LPairs& L, int P, const double* binom,
               const float2* utab, const float* lgtab, const double2* mp, float2* mp32,
               long nmp, double2* lo, int nlev, int* err_dev, cudaStream_t st) {
  if (L.npairs == 0) return IER_OK;
  if (nlev > 64 || !m2l_tc_supported(P)) return IER_BADARG;
  const int K = (P + 7) / 8 * 8, N = P <= 16 ? 16 : 32;
  const TcSmem S = tc_layout(P, K, N);
  size_t sm = S.total + 1024;  // room to align the base
  int dev = 0, nsm = 148;
  B2_CHECK(cudaGetDevice(&dev));
  B2_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  k_mp_to_f32<<<ceil_div(nmp, 256), 256, 0, st>>>(mp, nmp, mp32);
  B2_LAUNCH_CHECK();
  const int TP = TC_ROWS / ND;
  long ntiles = (L.npairs + TP - 1) / TP;
  int grid = (int)std::min<long>(ntiles, 3L * nsm);
  auto launch = [&](auto kern) {
    set_smem_attr(kern, sm);
    kern<<<grid, 128, sm, st>>>(L.pairs.p, L.npairs, P, N, binom, utab, lgtab, t.boxsize, nlev,
                                mp32, lo, err_dev);
    B2_LAUNCH_CHECK();
  };
#define B2_TC_K(NDV)                           \
  switch (K) {                                 \
    case 8: launch(k_m2l_tc<NDV, 8>); break;   \
    case 16: launch(k_m2l_tc<NDV, 16>); break; \
    case 24: launch(k_m2l_tc<NDV, 24>); break; \
    default: launch(k_m2l_tc<NDV, 32>); break; \
  }
  switch (ND) {
    case 8: B2_TC_K(8); break;
    case 4: B2_TC_K(4); break;
    case 2: B2_TC_K(2); break;
    default: B2_TC_K(1); break;
  }
#undef B2_TC_K
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
