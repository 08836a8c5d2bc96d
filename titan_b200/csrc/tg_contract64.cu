// FP64 chi0 contraction and epilogues.
//
// The 16 spin-block products of eintshechi.F90:86-104 are, for every site
// pair (i, j), one complex GEMM over the (k, E) points:
//
//   C_ij[u][v] = sum_p A_p[u] B_p[v],   u = (a1 nu, a2 gama), v = (b1 mu, b2 xi)
//
// with A_p = w_p G1_ij and B_p = (G2^T)_ij on the imaginary axis and
// A_p = w_p (G1 - G1^dagger)_ij, B_p = conj(G2)_ij on the real axis
// (eintshechi.F90:146-164).  The chi element is then picked out of C in the
// epilogue (chi = C_ij + conj(C_ji) with permuted indices, Fint = -i D_ij).
// This file holds the FP64 SIMT GEMM (the plain-precision GPU path), the
// chi assembly epilogue and a block-partial reduction.
#include "tg_internal.cuh"

#include <algorithm>

namespace tg {

namespace {

constexpr int TT = 16;            // thread grid side (TT x TT = 256 threads)
constexpr int PT = 7;             // complex entries per thread and dimension
constexpr int TILE = TT * PT;     // 112: three tiles cover 4*9*9 = 324 (sp-d sites)
constexpr int KC = 8;             // points per shared-memory stage
constexpr size_t kSmem = sizeof(double2) * 2 * 2 * KC * TILE;

__global__ void __launch_bounds__(TT * TT, 1)
gemm64_kernel(const double2* __restrict__ A, const double2* __restrict__ B, int64_t ld, int64_t np, int nsplit,
              const PairTile* __restrict__ tiles, const int* __restrict__ pair_M, const int* __restrict__ pair_aoff,
              const int64_t* __restrict__ pair_coff, double2* __restrict__ Cpart, int64_t cstride) {
  extern __shared__ __align__(16) double2 smem64[];
  double2 (*As)[KC][TILE] = reinterpret_cast<double2 (*)[KC][TILE]>(smem64);
  double2 (*Bs)[KC][TILE] = reinterpret_cast<double2 (*)[KC][TILE]>(smem64 + 2 * KC * TILE);
  const int tile_id = blockIdx.x / nsplit;
  const int split = blockIdx.x % nsplit;
  const PairTile t = tiles[tile_id];
  const int M = pair_M[t.pair];
  const int aoff = pair_aoff[t.pair];
  const int64_t p_begin = np * split / nsplit;
  const int64_t p_end = np * (split + 1) / nsplit;
  const int tid = threadIdx.x;
  const int ty = tid / TT, tx = tid % TT;

  double2 acc[PT][PT];
#pragma unroll
  for (int i = 0; i < PT; ++i)
#pragma unroll
    for (int j = 0; j < PT; ++j) acc[i][j] = make_double2(0.0, 0.0);

  auto load_stage = [&](int buf, int64_t p0) {
    // KC x TILE complex for A and for B; 16-byte cp.async per element
    for (int e = tid; e < KC * TILE; e += TT * TT) {
      const int kk = e / TILE, col = e % TILE;
      const int64_t p = p0 + kk;
      const int ua = t.u0 + col, vb = t.v0 + col;
      double2* da = &As[buf][kk][col];
      double2* db = &Bs[buf][kk][col];
      const bool pa = (p < p_end) && (ua < M);
      const bool pb = (p < p_end) && (vb < M);
      const double2* sa = pa ? A + p * ld + aoff + ua : A;
      const double2* sb = pb ? B + p * ld + aoff + vb : B;
      const unsigned sda = (unsigned)__cvta_generic_to_shared(da);
      const unsigned sdb = (unsigned)__cvta_generic_to_shared(db);
      const int na = pa ? 16 : 0, nb = pb ? 16 : 0;
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sda), "l"(sa), "r"(na));
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sdb), "l"(sb), "r"(nb));
    }
    asm volatile("cp.async.commit_group;\n" ::);
  };

  const int64_t nstages = (p_end - p_begin + KC - 1) / KC;
  if (nstages > 0) load_stage(0, p_begin);
  for (int64_t s = 0; s < nstages; ++s) {
    const int buf = (int)(s & 1);
    if (s + 1 < nstages) {
      load_stage(buf ^ 1, p_begin + (s + 1) * KC);
      asm volatile("cp.async.wait_group 1;\n" ::);
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < KC; ++kk) {
      double2 a[PT], b[PT];
#pragma unroll
      for (int i = 0; i < PT; ++i) a[i] = As[buf][kk][ty + TT * i];
#pragma unroll
      for (int j = 0; j < PT; ++j) b[j] = Bs[buf][kk][tx + TT * j];
#pragma unroll
      for (int i = 0; i < PT; ++i)
#pragma unroll
        for (int j = 0; j < PT; ++j) acc[i][j] = cfma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
  double2* C = Cpart + (int64_t)split * cstride + pair_coff[t.pair];
#pragma unroll
  for (int i = 0; i < PT; ++i) {
    const int u = t.u0 + ty + TT * i;
    if (u >= M) continue;
#pragma unroll
    for (int j = 0; j < PT; ++j) {
      const int v = t.v0 + tx + TT * j;
      if (v >= M) continue;
      double2* c = C + (int64_t)u * M + v;
      *c = cadd(*c, acc[i][j]);
    }
  }
}

// a(s): spin of the G1 side, b(s): spin of the G2 side for chi index s = 1..4
// (0 = up, 1 = down), read off the table of eintshechi.F90:86-104.
__device__ __forceinline__ int spin_a(int s) { return (s == 0 || s == 2) ? 1 : 0; }
__device__ __forceinline__ int spin_b(int s) { return (s >= 2) ? 1 : 0; }

__global__ void chi_epilogue_kernel(const double2* __restrict__ Cpart, const double2* __restrict__ Dpart, int nsplit,
                                    int64_t cstride, int dimens, const int* __restrict__ decode,
                                    const int* __restrict__ norb, const int64_t* __restrict__ pair_coff, int n_atoms,
                                    double scale, double2* __restrict__ chi) {
  const int64_t total = (int64_t)dimens * dimens;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int R = (int)(idx % dimens), Cc = (int)(idx / dimens);   // column-major (Fortran)
    const int dr = decode[R], dc = decode[Cc];
    const int s1 = dr & 3, i = (dr >> 2) & 1023, mu = (dr >> 12) & 63, nu = (dr >> 18) & 63;
    const int s2 = dc & 3, j = (dc >> 2) & 1023, ga = (dc >> 12) & 63, xi = (dc >> 18) & 63;
    const int ni = norb[i], nj = norb[j];
    const int a1 = spin_a(s1), b1 = spin_b(s1), a2 = spin_a(s2), b2 = spin_b(s2);
    // C_ij[(a1 nu, a2 gama), (b1 mu, b2 xi)]
    const int Mij = 4 * ni * nj;
    const int64_t u = (int64_t)(a1 * ni + nu) * (2 * nj) + (a2 * nj + ga);
    const int64_t v = (int64_t)(b1 * ni + mu) * (2 * nj) + (b2 * nj + xi);
    const int64_t off_ij = pair_coff[i * n_atoms + j] + u * Mij + v;
    // C_ji[(a2 gama, a1 nu), (b2 xi, b1 mu)]
    const int64_t u2 = (int64_t)(a2 * nj + ga) * (2 * ni) + (a1 * ni + nu);
    const int64_t v2 = (int64_t)(b2 * nj + xi) * (2 * ni) + (b1 * ni + mu);
    const int64_t off_ji = pair_coff[j * n_atoms + i] + u2 * Mij + v2;
    double2 c1 = make_double2(0, 0), c2 = c1, d = c1;
    for (int sp = 0; sp < nsplit; ++sp) {
      c1 = cadd(c1, Cpart[sp * cstride + off_ij]);
      c2 = cadd(c2, Cpart[sp * cstride + off_ji]);
      if (Dpart) d = cadd(d, Dpart[sp * cstride + off_ij]);
    }
    // chi_imag + Fint, Fint = -i D
    double2 val = cadd(c1, cconj(c2));
    val = cadd(val, make_double2(d.y, -d.x));
    chi[idx] = cscale(val, scale);
  }
}

__global__ void reduce_blocks_kernel(const double2* __restrict__ part, int nblocks, int len, double2* __restrict__ out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < len; e += gridDim.x * blockDim.x) {
    double2 s = make_double2(0, 0);
    for (int b = 0; b < nblocks; ++b) s = cadd(s, part[(int64_t)b * len + e]);
    out[e] = s;
  }
}

}  // namespace

cudaError_t launch_gemm64(const double2* A, const double2* B, int64_t ld, int64_t np, int nsplit,
                          const PairTile* tiles, int ntiles, const int* pair_M, const int* pair_aoff,
                          const int64_t* pair_coff, double2* Cpart, int64_t cstride, cudaStream_t s) {
  if (np <= 0 || ntiles <= 0) return cudaSuccess;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(gemm64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  gemm64_kernel<<<ntiles * nsplit, TT * TT, kSmem, s>>>(A, B, ld, np, nsplit, tiles, pair_M, pair_aoff, pair_coff,
                                                    Cpart, cstride);
  return cudaGetLastError();
}

cudaError_t launch_chi_epilogue(const double2* Cpart, const double2* Dpart, int nsplit, int64_t cstride,
                                int dimens, const int* decode, const int* norb, const int64_t* pair_coff,
                                int n_atoms, double scale, double2* chi, cudaStream_t s) {
  const int64_t total = (int64_t)dimens * dimens;
  int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  chi_epilogue_kernel<<<blocks, 256, 0, s>>>(Cpart, Dpart, nsplit, cstride, dimens, decode, norb, pair_coff,
                                             n_atoms, scale, chi);
  return cudaGetLastError();
}

cudaError_t launch_reduce_blocks(const double2* part, int nblocks, int len, double2* out, cudaStream_t s) {
  int blocks = (len + 255) / 256;
  if (blocks > 1024) blocks = 1024;
  if (blocks < 1) blocks = 1;
  reduce_blocks_kernel<<<blocks, 256, 0, s>>>(part, nblocks, len, out);
  return cudaGetLastError();
}

int gemm64_tile() { return TILE; }

}  // namespace tg
