// Split-precision chi0 contraction (int8 slices on the tcgen05 tensor cores).
//
// The contraction C_ij[u][v] = sum_p A_p[u] B_p[v] of a pass is evaluated on
// integers.  Per chunk c of points (a run of one energy, at most the context's
// chunk length, itself at most kSplitMaxChunk points) and per operand element e,
// a power-of-two scale 2^E[c][e] bounds max_p |Re|, |Im| of the element over the
// chunk; the element becomes the 46-bit integer X = rint(x 2^(46 - E)) held as six
// balanced base-256 digits (int8, most significant first; the top one in
// [-64, 64]).  The int8 tensor cores give exact int32 sums of digit products;
// products of digit pairs (i, j) (1-based) are accumulated per level L = i + j
// (L = 2..7, 21 products) in six TMEM accumulators, and every chunk end the levels
// are recombined in FP64 with weights 2^(4 - 8L) 2^(E_A + E_B) and added to the
// FP64 partial accumulators (same layout as the FP64 path).  Short chunks follow
// the magnitude of G along the k list, so that most points use most of the 46
// bits: near the real axis the error falls with the chunk length.
//
// Operand digits live in HBM as K-step blocks (32 points), K-major in the
// canonical no-swizzle core-matrix layout, so one bulk copy stages a block:
//   A block (t, gA): [slice 5][k half 2][row 128][16 B], rows 0..63 Re and
//                    64..127 Im of 64 complex rows u of one site pair
//   B block (t, gB): [slice 5][k half 2][row 80][16 B], rows 0..39 Re and
//                    40..79 Im of 40 complex columns v of one site pair
// One M=128 x N=80 x K=32 MMA per digit pair gives, for the 64 x 40 complex
// tile, the four real products Ar Br, Ar Bi, Ai Br, Ai Bi at once.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace tg {

constexpr int kSplitSlices = 6;        // base-256 digits per value
constexpr int kSplitBits = 46;         // |X| <= 2^46
constexpr int kSplitK = 32;            // points per K-step (one MMA K)
constexpr int kSplitRowsA = 64;        // complex rows per A group
constexpr int kSplitColsB = 40;        // complex columns per B group
constexpr int kSplitMaxChunk = 16384;  // points per chunk: level sums stay below 6 2^28 < 2^31
constexpr int kSplitABlock = kSplitSlices * 2 * kSplitRowsA * kSplitK;   // 24576 bytes
constexpr int kSplitBBlock = kSplitSlices * 2 * kSplitColsB * kSplitK;   // 15360 bytes

// one 64-row (A) or 40-column (B) group of a site pair's operand elements
struct SplitGroup {
  int elem0;    // first element (pair-block operand index)
  int nvalid;   // valid rows (the rest is zero padding)
};

// one output tile: A group gA x B group gB of pair `pair`
struct SplitTile {
  int pair, gA, gB, u0, v0;
};

// host-side split layout of a system (built once per tg_set_system)
struct SplitLayout {
  std::vector<SplitGroup> groupsA, groupsB;
  std::vector<SplitTile> tiles;
};

void split_build_layout(int n_pairs, const int* pair_M, const int* pair_aoff, SplitLayout& out);

// chunks of one pass: points sharing an energy, at most kSplitMaxChunk of them; point s
// of chunk c sits in slot slot0[c] + s * stride of the pass (stride 1 for a pass in mesh
// order, the number of energies for a k-major pass over a tabulated mesh)
struct SplitChunks {
  std::vector<int> slot0, count, kstart, kchunk;   // kstart has n_chunks + 1 entries
  int stride = 1;
  int n_ksteps() const { return kstart.empty() ? 0 : kstart.back(); }
  int n_chunks() const { return (int)count.size(); }
};

// device views used by the kernels
struct SplitPassDev {
  int n_chunks = 0, n_ksteps = 0;
  int stride = 1;
  const int* slot0 = nullptr;
  const int* count = nullptr;
  const int* kstart = nullptr;
  const int* kchunk = nullptr;
};

// per-element max |Re|, |Im| over each chunk, as the bit pattern of a non-negative
// double (M64[c * ld + e]; must start at zero)
cudaError_t split_rowmax(const double2* X, int64_t ld, const SplitPassDev& p, unsigned long long* M64,
                         cudaStream_t s);

// the same maxima (as the bits of 2^(E - 1), E the largest frexp exponent) from an int16
// exponent sidecar of the operand; ld must be even
cudaError_t split_rowmax_e16(const int16_t* E16, int64_t ld, const SplitPassDev& p, unsigned long long* M64,
                             cudaStream_t s);

// Quantisation bound of a pass (the chunk maxima M64 of both operands, before the next pass
// overwrites them): bnd[t] += sum_c count[c] ||2^E_A(c, t)|| ||2^E_B(c, t)|| per site pair t.
// Per point and real product the format's error is below 6.02 2^(E_A + E_B - 46): rounding to
// 46 bits, 2^(E_A + E_B - 46), plus the digit products of levels i + j >= 6 it drops,
// (5 2^46 + 2^40 + 3 2^30 + 2^23 + 2^14) 2^(E_A + E_B - 92) with balanced digits |d| <= 128.
cudaError_t split_bound(const unsigned long long* m64A, const unsigned long long* m64B, int64_t ld,
                        const SplitPassDev& p, const int* pair_M, const int* pair_aoff, int n_pairs, double* bnd,
                        cudaStream_t s);

// digits of one operand for a pass; writes E[c * ld + e] for every valid element
cudaError_t split_quantize(const double2* X, int64_t ld, const SplitPassDev& p, const SplitGroup* groups,
                           int n_groups, int rows, const unsigned long long* M64, int* E, int8_t* dig,
                           cudaStream_t s);

struct SplitContractArgs {
  const int8_t* A = nullptr;
  const int8_t* B = nullptr;
  int GA = 0, GB = 0;
  const SplitTile* tiles = nullptr;
  int ntiles = 0;
  int nsplit = 1;
  SplitPassDev pass;
  const int* EA = nullptr;
  const int* EB = nullptr;
  int64_t ld = 0;
  const int* pair_M = nullptr;
  const int* pair_aoff = nullptr;
  const int64_t* pair_coff = nullptr;
  double2* C = nullptr;        // partial accumulators, split s at C + s * cstride
  int64_t cstride = 0;
  int* err = nullptr;          // receives a non-zero code if a bounded wait gave up
  int num_ctas = 148;          // persistent CTAs (one per SM)
};

cudaError_t split_contract(const SplitContractArgs& a, cudaStream_t s);

// number of K-range splits for a tile count (balances waves over the SMs)
int split_nsplit(int ntiles, int num_sms, int64_t ksteps_hint);

}  // namespace tg
