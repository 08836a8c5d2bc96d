// Split-precision chi0 contraction on the tcgen05 tensor cores (int8 slices,
// exact int32 level sums in TMEM, FP64 recombination per chunk).
//
// Three kernels per pass and operand: split_rowmax_kernel (per chunk and
// element, the largest |Re|, |Im|), split_quantize_kernel (FP64 operand ->
// six int8 digit planes, K-step blocks) and split_contract_kernel (warp-
// specialised: one producer warp stages digit blocks with bulk copies into a
// five-stage shared-memory ring, one warp issues the 21 MMAs per K-step, eight
// warps drain the six int32 level accumulators from TMEM at every chunk end
// into FP64 sums held in registers until the unit ends).
// Every wait on an mbarrier is bounded (2 s of %globaltimer); on a timeout the
// kernel records an error code, waits (bounded) for its own copies and MMAs in
// flight, frees its TMEM and returns.
#include "tg_internal.cuh"
#include "tg_split.cuh"

#include <algorithm>
#include <cstdio>

namespace tg {

namespace {

// ----------------------------------------------------------------------------
// FP64 -> digits
// ----------------------------------------------------------------------------

constexpr int kRowmaxSlots = 64;

__global__ void split_rowmax_kernel(const double2* __restrict__ X, int64_t ld, int stride,
                                    const int* __restrict__ slot0, const int* __restrict__ count,
                                    unsigned long long* __restrict__ M64) {
  const int c = blockIdx.y;
  const int cnt = count[c];
  const int s_begin = blockIdx.x * kRowmaxSlots;
  if (s_begin >= cnt) return;
  const int s_end = min(cnt, s_begin + kRowmaxSlots);
  const int64_t base = (int64_t)slot0[c];
  for (int64_t e = threadIdx.x; e < ld; e += blockDim.x) {
    double m = 0.0;
    for (int s = s_begin; s < s_end; ++s) {
      const double2 v = X[(base + (int64_t)s * stride) * ld + e];
      m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
    }
    if (m > 0.0) atomicMax(&M64[(int64_t)c * ld + e], (unsigned long long)__double_as_longlong(m));
  }
}

// the same maxima from the exponent sidecar of the spectral G kernel (int16 per value,
// ld even): the largest exponent E of a chunk and element is stored as the bits of
// 2^(E - 1), whose frexp exponent is E, so the quantiser sees the scale it would get
// from the FP64 values; the pass reads 2 bytes per value instead of 16
__global__ void split_rowmax_e16_kernel(const int16_t* __restrict__ E16, int64_t ld, int stride,
                                        const int* __restrict__ slot0, const int* __restrict__ count,
                                        unsigned long long* __restrict__ M64) {
  const int c = blockIdx.y;
  const int cnt = count[c];
  const int s_begin = blockIdx.x * kRowmaxSlots;
  if (s_begin >= cnt) return;
  const int s_end = min(cnt, s_begin + kRowmaxSlots);
  const int64_t base = (int64_t)slot0[c];
  const int64_t ld2 = ld / 2;
  const uint32_t* W = reinterpret_cast<const uint32_t*>(E16);
  for (int64_t e2 = threadIdx.x; e2 < ld2; e2 += blockDim.x) {
    int m0 = -32768, m1 = -32768;
    for (int s = s_begin; s < s_end; ++s) {
      const uint32_t w = W[((base + (int64_t)s * stride) * ld) / 2 + e2];
      m0 = max(m0, (int)(int16_t)(w & 0xffffu));
      m1 = max(m1, (int)(int16_t)(w >> 16));
    }
    if (m0 > -32768)
      atomicMax(&M64[(int64_t)c * ld + 2 * e2], (unsigned long long)(m0 - 1 + 1023) << 52);
    if (m1 > -32768)
      atomicMax(&M64[(int64_t)c * ld + 2 * e2 + 1], (unsigned long long)(m1 - 1 + 1023) << 52);
  }
}

// Balanced base-256 digits of 16 integers |X| <= 2^46, slice-major: out[0] holds
// the top digits, out[1..5] the lower ones (most significant first).  With
// Y = X + 0x8080808080 the five lower balanced digits are bytes 0..4 of Y minus
// 128 (a byte-wise XOR with 0x80), and the top digit is Y >> 40 (in [-64, 64]).
__device__ __forceinline__ void digits16(const long long (&x)[16], uint4 (&out)[kSplitSlices]) {
  uint32_t lo[16], top[4] = {0u, 0u, 0u, 0u}, mid[4] = {0u, 0u, 0u, 0u};
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const long long y = x[k] + 0x8080808080LL;
    lo[k] = (uint32_t)y ^ 0x80808080u;
    mid[k >> 2] |= (((uint32_t)(y >> 32) & 255u) ^ 0x80u) << (8 * (k & 3));
    top[k >> 2] |= ((uint32_t)(int)(y >> 40) & 255u) << (8 * (k & 3));
  }
  uint32_t b[4][4];   // b[byte][group of four values]
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const uint32_t t0 = __byte_perm(lo[4 * j], lo[4 * j + 1], 0x5140);
    const uint32_t t1 = __byte_perm(lo[4 * j], lo[4 * j + 1], 0x7362);
    const uint32_t t2 = __byte_perm(lo[4 * j + 2], lo[4 * j + 3], 0x5140);
    const uint32_t t3 = __byte_perm(lo[4 * j + 2], lo[4 * j + 3], 0x7362);
    b[0][j] = __byte_perm(t0, t2, 0x5410);
    b[1][j] = __byte_perm(t0, t2, 0x7632);
    b[2][j] = __byte_perm(t1, t3, 0x5410);
    b[3][j] = __byte_perm(t1, t3, 0x7632);
  }
  out[0] = make_uint4(top[0], top[1], top[2], top[3]);
  out[1] = make_uint4(mid[0], mid[1], mid[2], mid[3]);
#pragma unroll
  for (int i = 2; i < kSplitSlices; ++i) out[i] = make_uint4(b[5 - i][0], b[5 - i][1], b[5 - i][2], b[5 - i][3]);
}

// Error bound of the format for one pass: for every site pair t (elements [aoff_t, aoff_t +
// M_t) of both operands) bnd[t] += sum_c count[c] ||s_A(c, t)||_2 ||s_B(c, t)||_2, with
// s_X(c, e) = 2^E the power of two above element e's maximum over chunk c (0 for a chunk of
// zeros).  A warp per (chunk, pair).
__device__ __forceinline__ double pow2_sq_above(unsigned long long bits) {
  const double m = __longlong_as_double((long long)bits);
  if (!(m > 0.0)) return 0.0;
  int E = 0;
  frexp(m, &E);
  return ldexp(1.0, 2 * E);
}

__global__ void split_bound_kernel(const unsigned long long* __restrict__ m64A,
                                   const unsigned long long* __restrict__ m64B, int64_t ld, int n_chunks,
                                   const int* __restrict__ count, const int* __restrict__ pair_M,
                                   const int* __restrict__ pair_aoff, int n_pairs, double* __restrict__ bnd) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int64_t items = (int64_t)n_chunks * n_pairs;
  for (int64_t it = blockIdx.x * (int64_t)nw + warp; it < items; it += (int64_t)gridDim.x * nw) {
    const int ch = (int)(it / n_pairs), t = (int)(it % n_pairs);
    const int M = pair_M[t];
    const int64_t base = (int64_t)ch * ld + pair_aoff[t];
    double sa = 0.0, sb = 0.0;
    for (int e = lane; e < M; e += 32) {
      sa += pow2_sq_above(m64A[base + e]);
      sb += pow2_sq_above(m64B[base + e]);
    }
    for (int o = 16; o > 0; o >>= 1) {
      sa += __shfl_xor_sync(0xffffffffu, sa, o);
      sb += __shfl_xor_sync(0xffffffffu, sb, o);
    }
    if (lane == 0 && sa > 0.0 && sb > 0.0) atomicAdd(bnd + t, (double)count[ch] * sqrt(sa) * sqrt(sb));
  }
}

// one thread per (K-step t, k half kc, group g, row r < rows): 16 points of one
// element, Re and Im parts
__global__ void __launch_bounds__(256) split_quantize_kernel(
    const double2* __restrict__ X, int64_t ld, int stride, int n_ksteps, const int* __restrict__ kchunk,
    const int* __restrict__ kstart, const int* __restrict__ slot0, const int* __restrict__ count,
    const SplitGroup* __restrict__ groups, int n_groups, int rows, const unsigned long long* __restrict__ M64,
    int* __restrict__ E, int8_t* __restrict__ dig) {
  const int64_t per_t = (int64_t)2 * n_groups * rows;
  const int64_t total = (int64_t)n_ksteps * per_t;
  const int64_t block_bytes = (int64_t)kSplitSlices * 2 * rows * kSplitK;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx % rows);
    const int g = (int)((idx / rows) % n_groups);
    const int kc = (int)((idx / ((int64_t)rows * n_groups)) % 2);
    const int t = (int)(idx / per_t);
    const int c = kchunk[t];
    const SplitGroup gr = groups[g];
    const int64_t e = gr.elem0 + r;
    // scale 2^(46 - E) with max |x| < 2^E; elements below 2^-977 of unit scale count as zero
    // (the scale's exponent field must stay below 2047)
    bool valid = r < gr.nvalid;
    int Ex = 0;
    if (valid) {
      const double m = __longlong_as_double((long long)M64[(int64_t)c * ld + e]);
      if (m > 0.0) frexp(m, &Ex);
      if (t == kstart[c] && kc == 0) E[(int64_t)c * ld + e] = Ex;
      if (m == 0.0 || Ex < -977) valid = false;
    }
    const double scale = __hiloint2double((1023 + kSplitBits - (valid ? Ex : 0)) << 20, 0);
    const int first = (t - kstart[c]) * kSplitK + kc * 16;   // point within the chunk
    const int cnt = count[c];
    const double2* src = X + ((int64_t)slot0[c] + (int64_t)first * stride) * ld + e;
    const int64_t step = (int64_t)stride * ld;
    long long xr[16], xi[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      double2 v = make_double2(0.0, 0.0);
      if (valid && first + k < cnt) v = src[k * step];
      xr[k] = __double2ll_rn(v.x * scale);
      xi[k] = __double2ll_rn(v.y * scale);
    }
    int8_t* blk = dig + ((int64_t)t * n_groups + g) * block_bytes + (int64_t)kc * 2 * rows * 16;
    uint4 d[kSplitSlices];
    digits16(xr, d);
#pragma unroll
    for (int i = 0; i < kSplitSlices; ++i)
      *reinterpret_cast<uint4*>(blk + (int64_t)i * 2 * rows * kSplitK + (int64_t)r * 16) = d[i];
    digits16(xi, d);
#pragma unroll
    for (int i = 0; i < kSplitSlices; ++i)
      *reinterpret_cast<uint4*>(blk + (int64_t)i * 2 * rows * kSplitK + (int64_t)(rows + r) * 16) = d[i];
  }
}

// ----------------------------------------------------------------------------
// tcgen05 contraction
// ----------------------------------------------------------------------------

constexpr int kMmaM = 128;
constexpr int kMmaN = 2 * kSplitColsB;     // 80
constexpr int kLevels = 6;                 // L = 2..7
constexpr int kStages = 5;
constexpr int kStageBytes = kSplitABlock + kSplitBBlock;   // 39936
constexpr int kHalfCols = kSplitColsB / 2;                 // complex columns per epilogue warp
constexpr int kXchBytes = 2 * 64 * 4 * 16 + 2 * 64 * 8;   // 2 halves x 64 rows x 4 complex, 2 x 40 column scales
constexpr int kEpiThreads = 256;                           // 8 epilogue warps
constexpr int kThreads = 64 + kEpiThreads;                 // producer, MMA, epilogue
constexpr uint32_t kTmemCols = 512;
constexpr int kBarOff = kStages * kStageBytes + kXchBytes;  // 8-byte aligned
constexpr int kNumBars = 2 * kStages + 3;
constexpr size_t kSplitSmem = 1024 + kBarOff + kNumBars * 8 + 16;
static_assert(kSplitSmem <= 232448, "the stage ring must fit the 227 KB of shared memory per CTA");
constexpr unsigned long long kWaitNs = 2000000000ull;        // 2 s per wait

__host__ __device__ constexpr uint32_t idesc_i8() {
  // c_format S32 (2), a/b format signed int8 (1), both K-major, N >> 3, M >> 4
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kMmaN >> 3) << 17) | ((uint32_t)(kMmaM >> 4) << 24);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;   // descriptor version of sm_100; layout type 0 = no swizzle
  return d;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait; false when the CTA aborted or 2 s passed (then sets the abort flag and err)
__device__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag, int* err, int code) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  uint32_t spins = 0;
  while (true) {
    if (mbar_try(bar, parity)) return true;
    if ((++spins & 255u) == 0) {
      if (*abort_flag) return false;
      if (global_ns() - t0 > kWaitNs) {
        *abort_flag = 1;
        atomicExch(err, code);
        return false;
      }
    }
  }
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

__device__ __forceinline__ void umma_i8(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, 256;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld4(uint32_t taddr, uint32_t (&v)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
               : "r"(taddr));
}

// 2^e for -1022 <= e <= 1023, from the bits
__device__ __forceinline__ double pow2(int e) { return __hiloint2double((1023 + e) << 20, 0); }

// exact double of an integer |v| < 2^51: its bits added to those of 1.5 * 2^52 give
// 1.5 * 2^52 + v (the same binade), and the subtraction is exact
__device__ __forceinline__ double i51_to_double(long long v) {
  return __longlong_as_double(v + 0x4338000000000000LL) - 6755399441055744.0;
}

// 2^28 sum_{L=2..7} S_L 2^(4 - 8L) for the six int32 level sums S_L of column k:
// hi = S_2 2^16 + S_3 2^8 + S_4 and lo = S_5 2^16 + S_6 2^8 + S_7 are exact integers
// below 2^48, and the value is hi + lo 2^-24 (one rounding)
__device__ __forceinline__ double levels_value(const uint32_t (&x)[kLevels][4], int k) {
  const long long hi = (long long)(int)x[0][k] * 65536LL + (long long)(int)x[1][k] * 256LL + (long long)(int)x[2][k];
  const long long lo = (long long)(int)x[3][k] * 65536LL + (long long)(int)x[4][k] * 256LL + (long long)(int)x[5][k];
  return fma(i51_to_double(lo), 0x1p-24, i51_to_double(hi));
}

// Persistent: CTA b takes the units (tile, K-range) b, b + gridDim.x, ...; units
// are numbered K-range-major so that the CTAs resident at one time share the
// digit blocks of one K-range in L2.  The stage ring and the drain count run
// on across units, so the producer prefetches the next unit while the
// epilogue drains the last one.
__global__ void __launch_bounds__(kThreads, 1) split_contract_kernel(SplitContractArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t raw_addr = (uint32_t)__cvta_generic_to_shared(smem_raw);
  const uint32_t base = (raw_addr + 1023u) & ~1023u;
  unsigned char* sbase = smem_raw + (base - raw_addr);
  const uint32_t bar0 = base + kBarOff;
  const uint32_t accfull = bar0 + 8u * (2 * kStages);
  const uint32_t accempty = accfull + 8u;
  const uint32_t flushbar = accfull + 16u;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sbase + kBarOff + kNumBars * 8);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sbase + kBarOff + kNumBars * 8 + 4);
  volatile int* epi_ok = reinterpret_cast<volatile int*>(sbase + kBarOff + kNumBars * 8 + 8);
  double2* xch = reinterpret_cast<double2*>(sbase + kStages * kStageBytes);   // [2][64 * 4]
  double* sbs = reinterpret_cast<double*>(sbase + kStages * kStageBytes + 2 * 64 * 4 * 16);   // [2][64]

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(bar0 + 8u * s, 1);
      mbar_init(bar0 + 8u * (kStages + s), 1);
    }
    mbar_init(accfull, 1);
    mbar_init(accempty, kEpiThreads);
    mbar_init(flushbar, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const int nunits = a.ntiles * a.nsplit;
  const int K = a.pass.n_ksteps;
  const int* kchunk = a.pass.kchunk;
  const int* kstart = a.pass.kstart;

  if (warp == 0) {
    // ---------------- producer: one lane stages digit blocks ----------------
    if (lane == 0) {
      uint32_t it = 0;
      uint32_t last_use[kStages];
      bool armed[kStages];
      for (int s = 0; s < kStages; ++s) armed[s] = false, last_use[s] = 0;
      bool ok = true;
      for (int un = blockIdx.x; un < nunits && ok; un += gridDim.x) {
        const int split = un / a.ntiles;
        const SplitTile tile = a.tiles[un % a.ntiles];
        const int k0 = (int)((int64_t)K * split / a.nsplit), k1 = (int)((int64_t)K * (split + 1) / a.nsplit);
        const int8_t* srcA = a.A + (int64_t)tile.gA * kSplitABlock;
        const int8_t* srcB = a.B + (int64_t)tile.gB * kSplitBBlock;
        for (int t = k0; t < k1; ++t, ++it) {
          const int s = (int)(it % kStages);
          const uint32_t use = it / kStages;
          if (use > 0 && !(ok = mbar_wait(bar0 + 8u * (kStages + s), (use - 1) & 1u, abort_flag, a.err, 1))) break;
          const uint32_t sa = base + (uint32_t)s * kStageBytes;
          const uint32_t fb = bar0 + 8u * s;
          mbar_expect_tx(fb, (uint32_t)kStageBytes);
          bulk_g2s(sa, srcA + (int64_t)t * a.GA * kSplitABlock, kSplitABlock, fb);
          bulk_g2s(sa + kSplitABlock, srcB + (int64_t)t * a.GB * kSplitBBlock, kSplitBBlock, fb);
          armed[s] = true;
          last_use[s] = use;
        }
      }
      if (!ok) {
        // let every copy this thread issued land before the CTA leaves
        for (int s = 0; s < kStages; ++s) {
          if (!armed[s]) continue;
          const uint64_t t0 = global_ns();
          while (!mbar_try(bar0 + 8u * s, last_use[s] & 1u) && global_ns() - t0 < kWaitNs) {
          }
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ---------------- MMA issuer: one lane ----------------
    if (lane == 0) {
      const uint32_t idesc = idesc_i8();
      uint32_t it = 0, d = 0;
      bool ok = true, issued = false;
      for (int un = blockIdx.x; un < nunits && ok; un += gridDim.x) {
        const int split = un / a.ntiles;
        const int k0 = (int)((int64_t)K * split / a.nsplit), k1 = (int)((int64_t)K * (split + 1) / a.nsplit);
        int t = k0;
        while (t < k1) {
          const int te = min(k1, kstart[kchunk[t] + 1]);
          if (d > 0) {
            if (!(ok = mbar_wait(accempty, (d - 1) & 1u, abort_flag, a.err, 2))) break;
            tc_fence_after();
          }
          for (int tt = t; tt < te; ++tt, ++it) {
            const int s = (int)(it % kStages);
            if (!(ok = mbar_wait(bar0 + 8u * s, (it / kStages) & 1u, abort_flag, a.err, 3))) break;
            tc_fence_after();
            const uint32_t sa = base + (uint32_t)s * kStageBytes;
            const uint32_t sb = sa + kSplitABlock;
            // digit pairs (i, j) (0-based) with level l = i + j <= 5, grouped by level: 21 MMAs
#pragma unroll
            for (int l = 0; l < kLevels; ++l) {
#pragma unroll
              for (int i = 0; i < kSplitSlices; ++i) {
                const int j = l - i;
                if (j < 0 || j >= kSplitSlices) continue;
                const bool first = i == (l > kSplitSlices - 1 ? l - (kSplitSlices - 1) : 0);
                const uint64_t ad =
                    smem_desc(sa + (uint32_t)i * (2 * kSplitRowsA * kSplitK), 2 * kSplitRowsA * 16, 128);
                const uint64_t bd =
                    smem_desc(sb + (uint32_t)j * (2 * kSplitColsB * kSplitK), 2 * kSplitColsB * 16, 128);
                umma_i8(tmem + (uint32_t)(l * kMmaN), ad, bd, idesc, (tt != t || !first) ? 1u : 0u);
              }
            }
            umma_commit(bar0 + 8u * (kStages + s));
            issued = true;
          }
          if (!ok) break;
          umma_commit(accfull);
          ++d;
          t = te;
        }
      }
      if (!ok && issued) {
        // wait for the MMAs already issued before TMEM is released
        umma_commit(flushbar);
        const uint64_t t0 = global_ns();
        while (!mbar_try(flushbar, 0) && global_ns() - t0 < kWaitNs) {
        }
      }
    }
    __syncwarp();
  } else {
    // ---------------- epilogue: warps 2..9 ----------------
    // Warp w reads TMEM lanes 32 (w % 4) .. + 31 (MMA rows: 0..63 Re A, 64..127 Im A of
    // complex row r % 64) and the half (w - 2) / 4 of the tile's 40 complex columns.  Each
    // thread keeps its row's FP64 sums for its 20 columns in registers over all chunks of a
    // unit: per chunk end it folds the six int32 levels into two exact 48-bit integers,
    // scales them by the chunk's power of two and adds; C is written once per unit.
    const int ep = threadIdx.x - 64;
    const int lane_base = 32 * (warp & 3);
    const int half = (warp - 2) >> 2;
    const int cbase = half * kHalfCols;
    const int r = lane_base + lane;
    const int part = r >> 6;
    const int rr = r & 63;
    uint32_t d = 0;
    bool ok = true;
    for (int un = blockIdx.x; un < nunits && ok; un += gridDim.x) {
      const int split = un / a.ntiles;
      const SplitTile tile = a.tiles[un % a.ntiles];
      const int k0 = (int)((int64_t)K * split / a.nsplit), k1 = (int)((int64_t)K * (split + 1) / a.nsplit);
      const int M = a.pair_M[tile.pair];
      const int64_t aoff = a.pair_aoff[tile.pair];
      const int u = tile.u0 + rr;
      double ax[kHalfCols], ay[kHalfCols];   // sums over the B real / imaginary columns
#pragma unroll
      for (int j = 0; j < kHalfCols; ++j) ax[j] = ay[j] = 0.0;
      int t = k0;
      while (t < k1) {
        const int c = kchunk[t];
        const int te = min(k1, kstart[c + 1]);
        // scales of the chunk, fetched while its MMAs still run (buffer d & 1 was last
        // read two chunks ago, before the accumulator barrier of the previous chunk): the
        // level fold times 2^(E_A - 14) 2^(E_B - 14) is the value (E >= -977, so both are
        // normal doubles and their product is exact)
        const int64_t erow = (int64_t)c * a.ld + aoff;
        double* sb = sbs + 64 * (d & 1u);
        if (ep < kSplitColsB) sb[ep] = pow2(tile.v0 + ep < M ? a.EB[erow + tile.v0 + ep] - 14 : 0);
        const double sa = pow2(u < M ? a.EA[erow + u] - 14 : 0);
        if (ep == 0) *epi_ok = mbar_wait(accfull, d & 1u, abort_flag, a.err, 4) ? 1 : 0;
        epi_sync();
        ok = *epi_ok != 0;
        epi_sync();
        if (!ok) break;
        tc_fence_after();
        const uint32_t trow = tmem + ((uint32_t)lane_base << 16) + (uint32_t)cbase;
#pragma unroll
        for (int g = 0; g < kHalfCols / 4; ++g) {
          uint32_t x[kLevels][4], y[kLevels][4];
#pragma unroll
          for (int l = 0; l < kLevels; ++l) {
            tmem_ld4(trow + (uint32_t)(l * kMmaN + 4 * g), x[l]);
            tmem_ld4(trow + (uint32_t)(l * kMmaN + kSplitColsB + 4 * g), y[l]);
          }
          tmem_wait_ld();
          if (g == kHalfCols / 4 - 1) {
            // every TMEM read of this thread has landed: the MMA warp may start the next chunk
            tc_fence_before();
            mbar_arrive(accempty);
          }
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const double sab = sa * sb[cbase + 4 * g + k];
            ax[4 * g + k] = fma(levels_value(x, k), sab, ax[4 * g + k]);
            ay[4 * g + k] = fma(levels_value(y, k), sab, ay[4 * g + k]);
          }
        }
        ++d;
        t = te;
      }
      if (!ok) break;
      // unit end: rows of part 0 hold (Ar Br, Ar Bi), rows of part 1 (Ai Br, Ai Bi) of the
      // same complex row; part 1 hands its sums over through shared memory, four columns at a time
      double2* xh = xch + half * 64 * 4;
      double2* Crow = a.C + (int64_t)split * a.cstride + a.pair_coff[tile.pair] + (int64_t)u * M;
#pragma unroll
      for (int g = 0; g < kHalfCols / 4; ++g) {
        if (part == 1) {
#pragma unroll
          for (int k = 0; k < 4; ++k) xh[rr * 4 + k] = make_double2(ax[4 * g + k], ay[4 * g + k]);
        }
        epi_sync();
        if (part == 0 && u < M) {
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const int v = tile.v0 + cbase + 4 * g + k;
            if (v >= M) continue;
            const double2 yy = xh[rr * 4 + k];
            double2 cv = Crow[v];
            cv.x += ax[4 * g + k] - yy.y;
            cv.y += ay[4 * g + k] + yy.x;
            Crow[v] = cv;
          }
        }
        epi_sync();
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
}

}  // namespace

void split_build_layout(int n_pairs, const int* pair_M, const int* pair_aoff, SplitLayout& out) {
  out.groupsA.clear();
  out.groupsB.clear();
  out.tiles.clear();
  for (int p = 0; p < n_pairs; ++p) {
    const int M = pair_M[p];
    const int gA0 = (int)out.groupsA.size(), gB0 = (int)out.groupsB.size();
    const int na = (M + kSplitRowsA - 1) / kSplitRowsA, nb = (M + kSplitColsB - 1) / kSplitColsB;
    for (int g = 0; g < na; ++g)
      out.groupsA.push_back(SplitGroup{pair_aoff[p] + g * kSplitRowsA, std::min(kSplitRowsA, M - g * kSplitRowsA)});
    for (int g = 0; g < nb; ++g)
      out.groupsB.push_back(SplitGroup{pair_aoff[p] + g * kSplitColsB, std::min(kSplitColsB, M - g * kSplitColsB)});
    for (int ga = 0; ga < na; ++ga)
      for (int gb = 0; gb < nb; ++gb)
        out.tiles.push_back(SplitTile{p, gA0 + ga, gB0 + gb, ga * kSplitRowsA, gb * kSplitColsB});
  }
}

int split_nsplit(int ntiles, int num_sms, int64_t ksteps_hint) {
  // cost of a split count: waves x (K-steps per unit + a drain and start-up of ~24 K-steps)
  int best = 1;
  double best_cost = 1e300;
  for (int s = 1; s <= 64; ++s) {
    const int64_t units = (int64_t)ntiles * s;
    const int64_t waves = (units + num_sms - 1) / num_sms;
    const double cost = (double)waves * ((double)ksteps_hint / s + 12.0);
    if (cost < best_cost * 0.999) {
      best_cost = cost;
      best = s;
    }
  }
  return best;
}

cudaError_t split_rowmax(const double2* X, int64_t ld, const SplitPassDev& p, unsigned long long* M64,
                         cudaStream_t s) {
  if (p.n_chunks <= 0) return cudaSuccess;
  const int gx = (kSplitMaxChunk + kRowmaxSlots - 1) / kRowmaxSlots;
  split_rowmax_kernel<<<dim3(gx, p.n_chunks), 256, 0, s>>>(X, ld, p.stride, p.slot0, p.count, M64);
  return cudaGetLastError();
}

cudaError_t split_rowmax_e16(const int16_t* E16, int64_t ld, const SplitPassDev& p, unsigned long long* M64,
                             cudaStream_t s) {
  if (p.n_chunks <= 0) return cudaSuccess;
  if (ld % 2) return cudaErrorInvalidValue;
  const int gx = (kSplitMaxChunk + kRowmaxSlots - 1) / kRowmaxSlots;
  split_rowmax_e16_kernel<<<dim3(gx, p.n_chunks), 256, 0, s>>>(E16, ld, p.stride, p.slot0, p.count, M64);
  return cudaGetLastError();
}

cudaError_t split_bound(const unsigned long long* m64A, const unsigned long long* m64B, int64_t ld,
                        const SplitPassDev& p, const int* pair_M, const int* pair_aoff, int n_pairs, double* bnd,
                        cudaStream_t s) {
  if (p.n_chunks <= 0 || n_pairs <= 0) return cudaSuccess;
  const int64_t warps = (int64_t)p.n_chunks * n_pairs;
  const int blocks = (int)std::min<int64_t>((warps + 7) / 8, 148 * 8);
  split_bound_kernel<<<blocks, 256, 0, s>>>(m64A, m64B, ld, p.n_chunks, p.count, pair_M, pair_aoff, n_pairs, bnd);
  return cudaGetLastError();
}

cudaError_t split_quantize(const double2* X, int64_t ld, const SplitPassDev& p, const SplitGroup* groups,
                           int n_groups, int rows, const unsigned long long* M64, int* E, int8_t* dig,
                           cudaStream_t s) {
  if (p.n_ksteps <= 0) return cudaSuccess;
  const int64_t total = (int64_t)p.n_ksteps * 2 * n_groups * rows;
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  split_quantize_kernel<<<blocks, 256, 0, s>>>(X, ld, p.stride, p.n_ksteps, p.kchunk, p.kstart, p.slot0, p.count, groups,
                                               n_groups, rows, M64, E, dig);
  return cudaGetLastError();
}

cudaError_t split_contract(const SplitContractArgs& a, cudaStream_t s) {
  if (a.pass.n_ksteps <= 0 || a.ntiles <= 0) return cudaSuccess;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e =
        cudaFuncSetAttribute(split_contract_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSplitSmem);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  const int grid = std::min(a.ntiles * a.nsplit, a.num_ctas > 0 ? a.num_ctas : 148);
  split_contract_kernel<<<grid, kThreads, kSplitSmem, s>>>(a);
  return cudaGetLastError();
}

}  // namespace tg
