// Internal declarations shared by the CUDA translation units of libtitan_gpu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace tg {

// ---------------------------------------------------------------------------
// complex FP64 helpers (double2 = re, im)
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ double2 cmk(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// acc + a*b
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 acc) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
  return acc;
}
// acc - a*b
__device__ __forceinline__ double2 cfms(double2 a, double2 b, double2 acc) {
  acc.x = fma(-a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(-a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
  return acc;
}
// 1/a with scaling against overflow
__device__ __forceinline__ double2 crecip(double2 a) {
  double s = fmax(fabs(a.x), fabs(a.y));
  if (s == 0.0) return make_double2(0.0, 0.0);
  double xr = a.x / s, yr = a.y / s;
  double den = s * (xr * xr + yr * yr);
  return make_double2(xr / den, -yr / den);
}

// Reciprocal of a positive double by Newton-Raphson: start from the
// hardware approximation (rcp.approx.ftz.f64, about 20 correct bits) and
// apply r <- r + r (1 - s r) three times (quadratic convergence, so well past
// 53 bits); the result is within a few ulp of 1/s.
__device__ __forceinline__ double rcp_newton(double s) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(s));
  double e = fma(-s, r, 1.0);
  r = fma(r, e, r);
  e = fma(-s, r, 1.0);
  r = fma(r, e, r);
  e = fma(-s, r, 1.0);
  r = fma(r, e, r);
  return r;
}

// 1/a = conj(a) / |a|^2 for pivots of moderate magnitude (|a|^2 well inside
// the double range, true for z - H(k) entries); returns 0 for a == 0.
__device__ __forceinline__ double2 crecip_fast(double2 a) {
  const double s = fma(a.x, a.x, a.y * a.y);
  if (s == 0.0) return make_double2(0.0, 0.0);
  const double r = rcp_newton(s);
  return make_double2(a.x * r, -a.y * r);
}

// ---------------------------------------------------------------------------
// Output transforms of the Green-function kernel
// ---------------------------------------------------------------------------
enum GreenMode : int {
  MODE_RAW = 0,       // G column-major per point (test hook)
  MODE_A_IMAG = 1,    // w * G, pair-block layout
  MODE_B_IMAG = 2,    // G^T, pair-block layout
  MODE_A_REAL = 3,    // w * (G - G^dagger), pair-block layout
  MODE_B_REAL = 4,    // conj(G), pair-block layout
  MODE_EXPECT = 5,    // accumulate diagonal site blocks (occupations / moments)
  MODE_GG = 6,        // accumulate the orbital-diagonal GG tensor (Jacobian)
  MODE_DIAG4 = 7,     // accumulate w * sigma-traces of diagonal orbitals (Fermi column)
  MODE_HK = 8,        // H(k) only (no inversion), column-major per point
  MODE_ENTRIES = 9,   // accumulate w * G(r_e, c_e) for a list of entries (gg_desc pairs, acc_len of them)
};

// A set of (k, z) points.  kind 0: flattened imaginary-axis list (y, kp, w per
// point).  kind 1: real axis, point p = nep * nk + ik with energy x2[nep],
// weight p2[nep] * w[ik], k = kp[ik].  kind 2: explicit (z, k) list (test hook).
struct PointSet {
  int kind = 0;
  const double* y = nullptr;
  const double* kp = nullptr;
  const double* w = nullptr;
  const double* x2 = nullptr;
  const double* p2 = nullptr;
  const double2* z = nullptr;
  int64_t nk = 0;
};

struct GreenArgs {
  PointSet pts;
  int64_t p0 = 0, np = 0;     // point range
  double zr = 0.0, zi = 0.0;  // z = (zr + x2) + i (zi + y)
  double q[3] = {0, 0, 0};
  int mode = MODE_RAW;
  // system
  int n = 0;                  // dimH
  int n_neigh = 0;
  const double* R = nullptr;  // [n_neigh][3]
  const int* pair_start = nullptr;   // [nat*nat+1]
  const int* pair_neigh = nullptr;   // [nblk]
  const double2* pair_t = nullptr;   // [nblk][nmax*nmax], t(or, oc) at oc*nmax + or
  int nmax = 0;
  int n_atoms = 0;
  const int* row_atom = nullptr;     // [n]
  const int* row_orb = nullptr;      // [n]
  const int* row_spin = nullptr;     // [n]
  const double2* h0 = nullptr;       // column-major n x n
  // outputs
  double2* out = nullptr;            // per-point operand / matrix
  double2* out2 = nullptr;           // optional second operand from the same inverse
  int mode2 = MODE_RAW;
  const int* outmap = nullptr;       // [n*n] row*n + col of pair-block slot o
  double2* acc = nullptr;            // per-CTA accumulators (EXPECT / GG / DIAG4)
  int acc_len = 0;                   // complex entries per CTA
  const int* gg_desc = nullptr;      // GG entry descriptors
  int* status = nullptr;             // first singular point (1-based), atomicMin
  // optional precomputed H(k) table (row-major n x n per k) with a k-major
  // traversal: work item wi -> k index wi / n_e, energy index wi % n_e
  const double2* htab = nullptr;
  int64_t n_e = 0;
  int64_t nk_tab = 0;
  const double* ylist = nullptr;     // imaginary parts of the energies (structured imaginary axis)
  // optional eigendecomposition of every k of the k-major traversal (spectral Green
  // functions; with or without htab): eigU[k][r][a] row-major, eigL[k][a];
  // outinv[r*n + c] = pair-block slot of (r, c)
  const double2* eigU = nullptr;
  const double* eigL = nullptr;
  // optional Householder tridiagonalisation of every k of the k-major traversal (dimensions
  // beyond the Jacobi kernel): T's diagonal triD[k][n] and off-diagonal triE[k][n], the rows
  // trirows[tri_ns] of Q as triQ[k][s][c]; the output is G over those rows and columns
  const double* triD = nullptr;
  const double* triE = nullptr;
  const double2* triQ = nullptr;
  const int* trirows = nullptr;
  int tri_ns = 0;
  const int* outinv = nullptr;
  // optional exponent sidecars of out / out2 (spectral G only): per stored value the
  // frexp exponent of max(|Re|, |Im|), -32768 for zero or subnormal
  int16_t* eout = nullptr;
  int16_t* eout2 = nullptr;
  // energy split of a tabulated imaginary-axis pass: y_side = +1 keeps the points with
  // Im z >= y_split (spectral kernel), -1 those below (one-warp Gauss-Jordan kernel); other
  // kernels ignore it and evaluate every point
  double y_split = 0.0;
  int y_side = 0;
  // device workspace of the kernels that exchange data through global memory (the
  // thread-block-cluster Gauss-Jordan kernel: green_cluster_ws_bytes)
  void* ws = nullptr;
  size_t ws_bytes = 0;
};

// true when launch_green evaluates these arguments with the spectral kernel (the only
// one that writes exponent sidecars)
bool green_is_spectral(const GreenArgs& a);

// Launch the fused H(k) + Gauss-Jordan kernel for any supported n.
// Returns cudaErrorInvalidValue for an unsupported dimension.
cudaError_t launch_green(const GreenArgs& a, int num_sms, cudaStream_t s, int* grid_used);
int green_supported(int n);
int green_warp_supported(int n, int mode);
cudaError_t launch_green_warp(const GreenArgs& a, int num_sms, cudaStream_t s, int* grid_used);
int green_w1_supported(int n, int mode);
cudaError_t launch_green_w1(const GreenArgs& a, int num_sms, cudaStream_t s, int* grid_used);
int green_acc_ctas(int n, int64_t np, int num_sms);
// any dimension up to 288, MODE_RAW only: one thread-block cluster per matrix
int green_cluster_supported(int n, int mode);
int green_cluster_size(int n);
size_t green_cluster_ws_bytes(int n, int num_sms);
cudaError_t launch_green_cluster(const GreenArgs& a, int num_sms, cudaStream_t s);

// FP64 pair-block contraction: Cpart[split][cpair_off + u*M + v] += sum_p A[p][off+u] B[p][off+v]
struct PairTile { int pair; int u0; int v0; };
cudaError_t launch_gemm64(const double2* A, const double2* B, int64_t ld, int64_t np, int nsplit,
                          const PairTile* tiles, int ntiles, const int* pair_M, const int* pair_aoff,
                          const int64_t* pair_coff, double2* Cpart, int64_t cstride, cudaStream_t s);

// chi assembly: chi(R, C) column-major from C/D partial sums.
cudaError_t launch_chi_epilogue(const double2* Cpart, const double2* Dpart, int nsplit, int64_t cstride,
                                int dimens, const int* decode, const int* norb, const int64_t* pair_coff,
                                int n_atoms, double scale, double2* chi, cudaStream_t s);

int gemm64_tile();
// H(k) table for a k list (plus q): H[k][r][c] = h0 + H_nl(k + q)
cudaError_t launch_hk_table(const GreenArgs& a, const double* kp, int64_t nk, const double* d_q, double2* phase_ws,
                            double2* H, cudaStream_t s);
cudaError_t launch_reduce_blocks(const double2* part, int nblocks, int len, double2* out, cudaStream_t s);

// Spectral Green functions: Jacobi eigendecomposition of an H(k) table and G from (U, lambda)
size_t eig_smem_bytes(int n);
int eig_supported(int n);
int eig_fast(int n);
cudaError_t launch_eig(const double2* H, int64_t nk, int n, double2* U, double* lam, int* status, int num_sms,
                       cudaStream_t s);
int spectral_supported(int mode, int mode2, bool has_out2);
// Resolvents from a Householder tridiagonalisation per k: H (an H(k) table, overwritten) ->
// T (D, E) and the rows `rows` of Q; G over those rows per point of a k-major pass (MODE_RAW)
int tri_supported(int n);
cudaError_t launch_tridiag(double2* H, int64_t nk, int n, const int* rows, int ns, double* D, double* E,
                           double2* Q, int num_sms, cudaStream_t s);
cudaError_t launch_green_tri(const GreenArgs& g, int num_sms, cudaStream_t s);
// per-CTA slices [grid][2 n] of the energy-summed diagonal spin blocks (uu, dd, ud, du per orbital)
cudaError_t launch_spec_expect(const double2* U, const double* lam, int64_t nk, int n, const double* ylist, int64_t n_e,
                               const double* w, double zr, double zi, const int* rows, double2* partial, int grid,
                               cudaStream_t s);
// out[ie][r] = -Im G_rr(e_ie + i eta) / pi summed over the tabulated k with weights w
cudaError_t launch_spec_ldos(const double2* U, const double* lam, const double* w, int64_t nk, int n,
                             const double* e, int n_e, double eta, double* out, int num_sms, cudaStream_t s);
cudaError_t launch_green_spectral(const GreenArgs& g, const double2* U, const double* lam, const int* outinv,
                                  int num_sms, cudaStream_t s);

// Linear SOC: X_p = G_p V G_p, and a column-major G_p into a pair-block operand layout
size_t gvg_smem_bytes(int n);
cudaError_t launch_gvg(const double2* G, const double2* V, int n, int64_t np, double2* X, int num_sms,
                       cudaStream_t s);
cudaError_t launch_operand(const double2* G, int n, int64_t np, int64_t p0, const PointSet& pts, int mode,
                           const int* outmap, double2* out, int num_sms, cudaStream_t s);
// operand of a Green-function launch g from its column-major G (MODE_RAW output of g):
// ld slots per point, outmap[o] = r * n + c (an orbital subset in pair-block order)
// eout (null: none): the operand's exponent sidecar (exponent_code16 of every value written)
cudaError_t launch_gather(const GreenArgs& g, const double2* G, int mode, const int* outmap, int64_t ld, double2* out,
                          int16_t* eout, int num_sms, cudaStream_t s);

// frexp exponent of max(|Re|, |Im|) from the bits (the exponent field - 1022 for a normal
// number), -32768 for zero or a subnormal: the exponent sidecar the split quantiser's row
// maxima read instead of the FP64 values
__device__ __forceinline__ int16_t exponent_code16(double2 v) {
  const double m = fmax(fabs(v.x), fabs(v.y));
  const int f = (int)((__double_as_longlong(m) >> 52) & 0x7ff);
  return f == 0 ? (int16_t)-32768 : (int16_t)(f - 1022);
}

// Exchange coupling: d-orbital GG tensors T(G(k), G(k - q)) and T(G(k - q), G(k)) per site pair
cudaError_t launch_jij(const double2* Ga, const double2* Gb, int64_t p0, int64_t np, const double* w, int n,
                       int n_atoms, const int* ia, const int* norb, const int* dstart, const int* dlist,
                       double2* partial, int grid, cudaStream_t s);

// Disturbance-response vertex (eintshe): one launch per pass over RAW G1 / G2
struct SheLaunch {
  const GreenArgs* g = nullptr;   // system tables (n, neighbours, hopping blocks)
  const double2* G1 = nullptr;
  const double2* G2 = nullptr;
  int64_t p0 = 0, np = 0;
  PointSet pts;
  int real_axis = 0;
  int dimens = 0;
  const int* tab = nullptr;       // [4][n / 2]
  const int* ia = nullptr;
  const int* norb = nullptr;
  const int* decode = nullptr;
  // register-tiled second stage: 3 x 3 tiles of the (sigma, s', site) output blocks, code
  // sigma | s' << 2 | site << 4 | x0 << 14 | y0 << 20, and the first df row of each site
  const int* ztiles = nullptr;
  int n_ztiles = 0;
  const int* rowoff = nullptr;
  double ue[3] = {0, 0, 0};
  unsigned char spins[3][16] = {};
  double2* partial = nullptr;     // [grid][4 dimens]
  int grid = 0;
  // k-major point order of a tabulated pass (n_e > 0): point p0 + pl -> k = klist[p / n_e],
  // energy p % n_e, as the inversion kernels walk an H(k) table
  int64_t n_e = 0, nk_tab = 0;
  const double* klist = nullptr;
};
// (n_ztiles: second-stage tiles of the system, 16 sum_i ceil(n_i / 3)^2)
size_t she_smem_bytes(int n, int dimens, int n_neigh, int n_ztiles);
// CTAs of one vertex launch (SMs x resident CTAs); 0 when the shared memory does not fit
int she_grid(int n, int dimens, int n_neigh, int n_ztiles, int num_sms);
cudaError_t launch_she(const SheLaunch& l, cudaStream_t s);
cudaError_t launch_she_prefactor(const double2* P, const double2* df, int dimens, double scale, double2* out,
                                 cudaStream_t s);

}  // namespace tg
