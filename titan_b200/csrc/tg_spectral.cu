// Spectral Green functions on tabulated k meshes.
//
// When every energy of a pass uses the same k list (uniform imaginary-axis
// meshes, the real-axis BZ), one H(k) serves every (E, k) point of that k.
// H(k) is Hermitian, H = U diag(lambda) U^+, so for every z at once
//   G(k, z) = (z - H(k))^-1 = U diag(1 / (z - lambda)) U^+,
// which for a block of energies is one GEMM with K = dimH:
//   G[z][(r, c)] = sum_a D[z][a] P[a][(r, c)],   D[z][a] = 1 / (z - lambda_a),
//   P[a][(r, c)] = U[r][a] conj(U[c][a]).
// The GEMM runs on the FP64 tensor cores (mma.sync m8n8k4 .f64; tcgen05 has no
// FP64 kind); P is formed on the fly from U in shared memory.  The same form
// gives G - G^+ with D = 2 i Im(1 / (z - lambda)).
//
// The eigendecomposition is a cyclic two-sided Jacobi iteration, one CTA per
// matrix, n / 2 disjoint rotations per step in round-robin order, sweeps until
// the off-diagonal Frobenius norm is below 1e-17 of the matrix norm (couplings
// under 1e-16 of it are zeroed without a rotation, see below).  A is kept
// exactly Hermitian (only the upper 2 x 2 blocks are rotated, the lower ones are
// their conjugates): a rounding-level anti-Hermitian part would survive every
// unitary rotation and stall the off-diagonal norm near eps.  Its
// backward error (H + dH = U Lambda U^+, |dH| ~ eps |H|, U unitary to eps) is of
// the same order as Gauss-Jordan's, so G agrees with the inverse to roundoff
// times |H| / dist(z, spectrum).  A post-pass re-orthonormalises U (one Newton-Schulz
// step) and takes the eigenvalues as Rayleigh quotients of H.  It costs a few
// inversions per k and is shared by all energies and frequencies of the k.
#include "tg_internal.cuh"

#include <algorithm>

namespace tg {

namespace {

constexpr int kEigThreads = 256;
constexpr int kEigMaxSweeps = 30;
constexpr int kSpecZ = 16;          // energies per task (two m8 fragments)
constexpr int kSpecThreads = 256;

// --------------------------------------------------------------------------- Jacobi
struct Rot {
  double c, s;
  double2 e;   // b / |b| of the rotated pair (1 when b = 0)
};

// pair k of round s of the circle schedule on n (even) indices: every pair once per n - 1 rounds
__device__ __forceinline__ void rr_pair(int s, int k, int n, int& p, int& q) {
  const int m = n - 1;
  if (k == 0) {
    p = s;
    q = m;
  } else {
    p = (s + k) % m;
    q = (s - k + m) % m;
  }
}

__device__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
  return t;
}

// The Hermitian working matrix A in shared memory: the full n x n array, or (PACKED, for n
// whose A and U do not both fit) the upper triangle only, column by column:
// A(i, j), i <= j, at j (j + 1) / 2 + i; A(j, i) = conj A(i, j).
template <bool PACKED>
struct HermA {
  double2* a;
  int n;
  __device__ __forceinline__ double2 get(int i, int j) const {
    if (!PACKED) return a[i * n + j];
    return i <= j ? a[j * (j + 1) / 2 + i] : cconj(a[i * (i + 1) / 2 + j]);
  }
  // A(i, j) = v and A(j, i) = conj v
  __device__ __forceinline__ void set(int i, int j, double2 v) const {
    if (!PACKED) {
      a[i * n + j] = v;
      a[j * n + i] = cconj(v);
    } else if (i <= j) {
      a[j * (j + 1) / 2 + i] = v;
    } else {
      a[i * (i + 1) / 2 + j] = cconj(v);
    }
  }
  __device__ __forceinline__ void set_diag(int i, double v) const {
    a[PACKED ? i * (i + 1) / 2 + i : i * n + i] = make_double2(v, 0.0);
  }
  __device__ __forceinline__ static int64_t entries(int n) { return PACKED ? (int64_t)n * (n + 1) / 2 : (int64_t)n * n; }
  // (i, j) of storage entry e (i <= j when PACKED)
  __device__ __forceinline__ void ij(int e, int& i, int& j) const {
    if (!PACKED) {
      i = e / n;
      j = e % n;
      return;
    }
    j = (int)((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);
    while (j * (j + 1) / 2 > e) --j;
    while ((j + 1) * (j + 2) / 2 <= e) ++j;
    i = e - j * (j + 1) / 2;
  }
};

constexpr int kEigCols = 3;   // columns per lane of the post-pass row products: n <= 96

// H: [nk][n][n] row-major (the H(k) table); U: [nk][n][n] row-major U[r][a]; lam: [nk][n]
template <bool PACKED>
__global__ void __launch_bounds__(kEigThreads) eig_jacobi_kernel(const double2* __restrict__ H, int64_t nk, int n,
                                                                 double2* __restrict__ Uout, double* __restrict__ lam,
                                                                 int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int np = n / 2;
  const int64_t na = HermA<PACKED>::entries(n);
  const HermA<PACKED> A{reinterpret_cast<double2*>(smem), n};
  double2* U = A.a + na;
  Rot* rot = reinterpret_cast<Rot*>(U + n * n);
  double* red = reinterpret_cast<double*>(rot + np);
  for (int64_t k = blockIdx.x; k < nk; k += gridDim.x) {
    // A = (H + H^+) / 2: the table's H(k) is Hermitian up to rounding; the iteration keeps
    // A exactly Hermitian (upper blocks computed, lower blocks their conjugates)
    const double2* Hk = H + k * (int64_t)n * n;
    for (int e = threadIdx.x; e < na; e += blockDim.x) {
      int r, c;
      A.ij(e, r, c);
      const double2 x = Hk[r * n + c], y = Hk[c * n + r];
      A.a[e] = r == c ? make_double2(x.x, 0.0) : make_double2(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
    }
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) U[e] = make_double2(e / n == e % n ? 1.0 : 0.0, 0.0);
    __syncthreads();
    bool converged = false;
    for (int sweep = 0; sweep < kEigMaxSweeps; ++sweep) {
      double off = 0.0, tot = 0.0;
      for (int e = threadIdx.x; e < na; e += blockDim.x) {
        int r, c;
        A.ij(e, r, c);
        // a stored off-diagonal entry of the packed form stands for two of the matrix
        const double m2 = (A.a[e].x * A.a[e].x + A.a[e].y * A.a[e].y) * (PACKED && r != c ? 2.0 : 1.0);
        tot += m2;
        if (r != c) off += m2;
      }
      off = block_sum(off, red);
      tot = block_sum(tot, red);
      if (off <= 1e-34 * tot) {
        converged = true;
        break;
      }
      // couplings below 1e-16 |A|_F are set to zero without a rotation (a backward error
      // below rounding): rotating them would turn the rounding noise inside a cluster of
      // degenerate eigenvalues into large random angles that undo the annihilation of the
      // couplings between clusters (linear instead of quadratic convergence)
      const double thr_b = 1e-16 * sqrt(tot);
      for (int s = 0; s < n - 1; ++s) {
        for (int kk = threadIdx.x; kk < np; kk += blockDim.x) {
          int p, q;
          rr_pair(s, kk, n, p, q);
          const double a = A.get(p, p).x, d = A.get(q, q).x;
          const double2 b = A.get(p, q);
          const double ab = hypot(b.x, b.y);
          Rot r;
          if (ab <= thr_b) {
            r.c = 1.0;
            r.s = 0.0;
            r.e = make_double2(1.0, 0.0);
          } else {
            const double tau = (d - a) / (2.0 * ab);
            const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + hypot(1.0, tau));
            r.c = 1.0 / sqrt(1.0 + t * t);
            r.s = t * r.c;
            r.e = make_double2(b.x / ab, b.y / ab);
          }
          rot[kk] = r;
        }
        __syncthreads();
        // A <- J^+ A J on 2 x 2 blocks (rows of pair k1, columns of pair k2), in place:
        // J = [[c, s], [-s conj(e), c conj(e)]] on (p, q); block (k2, k1) is the conjugate
        // transpose of block (k1, k2), written by the same thread
        for (int blk = threadIdx.x; blk < np * np; blk += blockDim.x) {
          const int k1 = blk / np, k2 = blk % np;
          if (k1 > k2) continue;
          int p1, q1, p2, q2;
          rr_pair(s, k1, n, p1, q1);
          rr_pair(s, k2, n, p2, q2);
          const Rot r1 = rot[k1], r2 = rot[k2];
          if (k1 == k2) {
            const double a = A.get(p1, p1).x, d = A.get(q1, q1).x;
            const double2 b = A.get(p1, q1);
            const double ab = hypot(b.x, b.y);
            const double t = r1.s / r1.c;
            A.set_diag(p1, a - t * ab);
            A.set_diag(q1, d + t * ab);
            A.set(p1, q1, make_double2(0.0, 0.0));
            continue;
          }
          const double2 xpp = A.get(p1, p2), xpq = A.get(p1, q2), xqp = A.get(q1, p2), xqq = A.get(q1, q2);
          const double2 e2c = cconj(r2.e);
          // X = A_blk J2
          const double2 ypq = cmul(e2c, xpq), yqq = cmul(e2c, xqq);
          const double2 x00 = csub(cscale(xpp, r2.c), cscale(ypq, r2.s));
          const double2 x01 = cadd(cscale(xpp, r2.s), cscale(ypq, r2.c));
          const double2 x10 = csub(cscale(xqp, r2.c), cscale(yqq, r2.s));
          const double2 x11 = cadd(cscale(xqp, r2.s), cscale(yqq, r2.c));
          // J1^+ X: rows (c x0 - s e x1, s x0 + c e x1)
          const double2 z10 = cmul(r1.e, x10), z11 = cmul(r1.e, x11);
          A.set(p1, p2, csub(cscale(x00, r1.c), cscale(z10, r1.s)));
          A.set(p1, q2, csub(cscale(x01, r1.c), cscale(z11, r1.s)));
          A.set(q1, p2, cadd(cscale(x00, r1.s), cscale(z10, r1.c)));
          A.set(q1, q2, cadd(cscale(x01, r1.s), cscale(z11, r1.c)));
        }
        // U <- U J (columns p, q of every row)
        for (int e = threadIdx.x; e < n * np; e += blockDim.x) {
          const int r = e / np, kk = e % np;
          int p, q;
          rr_pair(s, kk, n, p, q);
          const Rot rr = rot[kk];
          const double2 up = U[r * n + p], uq = cmul(cconj(rr.e), U[r * n + q]);
          U[r * n + p] = csub(cscale(up, rr.c), cscale(uq, rr.s));
          U[r * n + q] = cadd(cscale(up, rr.s), cscale(uq, rr.c));
        }
        __syncthreads();
      }
    }
    if (!converged && threadIdx.x == 0 && status) atomicMin(status, (int)(k < 0x7ffffffe ? k + 1 : 0x7fffffff));
    // Post-pass.  The accumulated rotations leave U unitary only to ~1e-14 and the diagonal of
    // the rotated A carries the rounding of every sweep; re-orthonormalised vectors and
    // Rayleigh-quotient eigenvalues together bring spectral occupations to the inversion's
    // accuracy (checked on a CPU emulation of this kernel: 1.3e-14 -> 4.4e-16 on Fe bcc).
    //  (1) E = U^H U - 1 into A (the rotated matrix is no longer needed; E is Hermitian)
    __syncthreads();
    for (int e = threadIdx.x; e < na; e += blockDim.x) {
      int i, j;
      A.ij(e, i, j);
      double2 acc = make_double2(i == j ? -1.0 : 0.0, 0.0);
      for (int r = 0; r < n; ++r) acc = cfma(cconj(U[r * n + i]), U[r * n + j], acc);
      A.a[e] = acc;
    }
    __syncthreads();
    //  (2) one Newton-Schulz step U <- U (1 - E / 2): a warp per row, the row read before written
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    for (int r = warp; r < n; r += nwarps) {
      double2 v[kEigCols];
#pragma unroll
      for (int m = 0; m < kEigCols; ++m) {
        v[m] = make_double2(0.0, 0.0);
        const int j = lane + 32 * m;
        if (j < n)
          for (int i = 0; i < n; ++i) v[m] = cfma(U[r * n + i], A.get(i, j), v[m]);
      }
      __syncwarp();
#pragma unroll
      for (int m = 0; m < kEigCols; ++m) {
        const int j = lane + 32 * m;
        if (j < n) U[r * n + j] = csub(U[r * n + j], cscale(v[m], 0.5));
      }
      __syncwarp();
    }
    __syncthreads();
    //  (3) lambda_a = Re u_a^H Hs u_a with Hs = (H + H^H) / 2 from the table
    for (int e = threadIdx.x; e < na; e += blockDim.x) {
      int r, c;
      A.ij(e, r, c);
      const double2 x = Hk[r * n + c], y = Hk[c * n + r];
      A.a[e] = r == c ? make_double2(x.x, 0.0) : make_double2(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
    }
    __syncthreads();
    double2* Uk = Uout + k * (int64_t)n * n;
    if (!PACKED) {
      // W = Hs U row by row into A (a warp per row, in place), then one thread per eigenvalue
      for (int r = warp; r < n; r += nwarps) {
        double2 v[kEigCols];
#pragma unroll
        for (int m = 0; m < kEigCols; ++m) {
          v[m] = make_double2(0.0, 0.0);
          const int j = lane + 32 * m;
          if (j < n)
            for (int c = 0; c < n; ++c) v[m] = cfma(A.a[r * n + c], U[c * n + j], v[m]);
        }
        __syncwarp();
#pragma unroll
        for (int m = 0; m < kEigCols; ++m) {
          const int j = lane + 32 * m;
          if (j < n) A.a[r * n + j] = v[m];
        }
        __syncwarp();
      }
      __syncthreads();
      for (int e = threadIdx.x; e < n * n; e += blockDim.x) Uk[e] = U[e];
      for (int a = threadIdx.x; a < n; a += blockDim.x) {
        double l = 0.0;
        for (int r = 0; r < n; ++r) {
          const double2 u = U[r * n + a], w = A.a[r * n + a];
          l = fma(u.x, w.x, fma(u.y, w.y, l));   // Re(conj(u) w)
        }
        lam[k * n + a] = l;
      }
    } else {
      // no room for W: a warp per eigenvalue, lanes over the rows r of sum_r conj(u_r) (Hs u)_r
      for (int e = threadIdx.x; e < n * n; e += blockDim.x) Uk[e] = U[e];
      for (int a = warp; a < n; a += nwarps) {
        double l = 0.0;
        for (int r = lane; r < n; r += 32) {
          double2 w = make_double2(0.0, 0.0);
          for (int c = 0; c < n; ++c) w = cfma(A.get(r, c), U[c * n + a], w);
          const double2 u = U[r * n + a];
          l = fma(u.x, w.x, fma(u.y, w.y, l));
        }
        for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
        if (lane == 0) lam[k * n + a] = l;
      }
    }
    __syncthreads();
  }
}

// --------------------------------------------------------------------------- G from (U, lambda)
// not volatile: the scheduler may interleave the MMAs of independent accumulators (a chain on
// one accumulator keeps its order through the data dependence, so results do not change)
__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

struct SpecArgs {
  GreenArgs g;
  const double2* U = nullptr;   // [nk][n][n]
  const double* lam = nullptr;  // [nk][n]
  const int* outinv = nullptr;  // [n*n] pair-block slot of (r, c) = r * n + c
  int kp = 0;                   // K padded to a multiple of 4
};

__host__ __device__ inline size_t spec_smem(int n, int kp) {
  return sizeof(double2) * ((size_t)n * kp + (size_t)kSpecZ * kp) + sizeof(double) * kSpecZ + sizeof(int) * kSpecZ;
}

// (row, col) of G that lands in output slot o for a mode
__device__ __forceinline__ void slot_rc(const SpecArgs& sa, int mode, int o, int& r, int& c) {
  const int n = sa.g.n;
  if (mode == MODE_RAW) {
    r = o % n;
    c = o / n;
    return;
  }
  const int rc = sa.g.outmap[o];
  if (mode == MODE_B_IMAG) {   // G^T
    c = rc / n;
    r = rc % n;
  } else {
    r = rc / n;
    c = rc % n;
  }
}

// frexp exponent of max(|Re|, |Im|) read from the bits (exponent field - 1022 for a
// normal number); zero and subnormal values give -32768
__device__ __forceinline__ int16_t exponent_code(double2 v) {
  const double m = fmax(fabs(v.x), fabs(v.y));
  const int f = (int)((__double_as_longlong(m) >> 52) & 0x7ff);
  return f == 0 ? (int16_t)-32768 : (int16_t)(f - 1022);
}

// five CTAs per SM (the occupancy its ~30 KB of shared memory allows at n = 36): 48
// registers with a 4-byte spill, measured faster than 64 registers at four CTAs
// ANTI (MODE_A_REAL, w (G - G^+)): the diagonal -2i y / |z - lambda|^2 is purely
// imaginary, so two of the four DMMAs per step would multiply by zero and are skipped
// THREADS = 1024 (one CTA per SM) where the shared memory of U leaves room for one CTA only
// (n > 72): 32 warps instead of 8 hide the DMMA and shared-memory latencies
template <bool ANTI, int THREADS>
__global__ void __launch_bounds__(THREADS, THREADS == kSpecThreads ? 5 : 1) spec_green_kernel(SpecArgs sa) {
  extern __shared__ __align__(16) unsigned char smem[];
  const GreenArgs& a = sa.g;
  const int n = a.n, kp = sa.kp, nn = n * n;
  double2* Us = reinterpret_cast<double2*>(smem);          // [n][kp]
  double2* Ds = Us + (size_t)n * kp;                        // [kSpecZ][kp]
  double* ws = reinterpret_cast<double*>(Ds + (size_t)kSpecZ * kp);
  int* item = reinterpret_cast<int*>(ws + kSpecZ);          // pass-local point of each row, -1 = none
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarp = blockDim.x >> 5;
  const int64_t ne = a.n_e;
  const int64_t per_k = (ne + kSpecZ - 1) / kSpecZ;
  const int64_t ik0 = a.p0 / ne, ik1 = (a.p0 + a.np - 1) / ne;
  const int64_t ntask = (ik1 - ik0 + 1) * per_k;
  const bool anti = ANTI;
  for (int64_t t = blockIdx.x; t < ntask; t += gridDim.x) {
    const int64_t ik = ik0 + t / per_k;
    const int64_t ie0 = (t % per_k) * kSpecZ;
    // rows of this task
    if (threadIdx.x < kSpecZ) {
      const int64_t ie = ie0 + threadIdx.x;
      const int64_t wi = ik * ne + ie;
      const bool kept = a.y_side <= 0 || a.pts.kind != 0 || (ie < ne && a.zi + a.ylist[ie] >= a.y_split);
      item[threadIdx.x] = (ie < ne && wi >= a.p0 && wi < a.p0 + a.np && kept) ? (int)(wi - a.p0) : -1;
    }
    const double2* Uk = sa.U + ik * (int64_t)nn;
    for (int e = threadIdx.x; e < n * kp; e += blockDim.x) {
      const int r = e / kp, aa = e % kp;
      Us[e] = aa < n ? Uk[r * n + aa] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    // D[z][a] and the weights
    const double* lk = sa.lam + ik * n;
    for (int e = threadIdx.x; e < kSpecZ * kp; e += blockDim.x) {
      const int zr = e / kp, aa = e % kp;
      double2 dv = make_double2(0.0, 0.0);
      if (item[zr] >= 0 && aa < n) {
        const int64_t ie = ie0 + zr;
        double x, y;
        if (a.pts.kind == 0) {
          x = a.zr;
          y = a.zi + a.ylist[ie];
        } else {
          x = a.zr + a.pts.x2[ie];
          y = a.zi;
        }
        x -= lk[aa];
        const double s = x * x + y * y;
        if (s == 0.0) {
          if (a.status) {
            const int64_t pidx = a.p0 + item[zr] + 1;
            atomicMin(a.status, (int)(pidx < 0x7fffffff ? pidx : 0x7fffffff));
          }
        } else {
          const double inv = 1.0 / s;
          dv = anti ? make_double2(0.0, -2.0 * y * inv) : make_double2(x * inv, -y * inv);
        }
      }
      Ds[e] = dv;
    }
    if (threadIdx.x < kSpecZ) {
      double w = 0.0;
      if (item[threadIdx.x] >= 0) {
        const int64_t ie = ie0 + threadIdx.x;
        w = a.pts.kind == 0 ? a.pts.w[ie * a.nk_tab + ik] : a.pts.p2[ie] * a.pts.w[ik];
      }
      ws[threadIdx.x] = w;
    }
    __syncthreads();
    // G tiles: 16 energies x 8 output slots per warp step
    const int g8 = lane >> 2, t4 = lane & 3;
    const int nfrag = (nn + 7) / 8;
    for (int nf = warp; nf < nfrag; nf += nwarp) {
      int rb = 0, cb = 0;
      const int ob = nf * 8 + g8;
      if (ob < nn) slot_rc(sa, a.mode, ob, rb, cb);
      const double2* ur = Us + (size_t)rb * kp;
      const double2* uc = Us + (size_t)cb * kp;
      double cr[2][2] = {{0.0, 0.0}, {0.0, 0.0}}, ci[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
      for (int k0 = 0; k0 < kp; k0 += 4) {
        const int ka = k0 + t4;
        const double2 pv = cmul(ur[ka], cconj(uc[ka]));
#pragma unroll
        for (int mf = 0; mf < 2; ++mf) {
          const double2 dv = Ds[(mf * 8 + g8) * kp + ka];
          if (!ANTI) dmma(cr[mf][0], cr[mf][1], dv.x, pv.x);
          dmma(cr[mf][0], cr[mf][1], -dv.y, pv.y);
          if (!ANTI) dmma(ci[mf][0], ci[mf][1], dv.x, pv.y);
          dmma(ci[mf][0], ci[mf][1], dv.y, pv.x);
        }
      }
#pragma unroll
      for (int mf = 0; mf < 2; ++mf) {
        const int zr = mf * 8 + g8;
        const int pl = item[zr];
        if (pl < 0) continue;
        const double w = ws[zr];
        // the lane's two slots are adjacent (nn is even): one 4-byte store of both exponents
        const int o0 = nf * 8 + 2 * t4;
        uint32_t codes = 0;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int o = o0 + j;
          if (o >= nn) continue;
          const double2 v = make_double2(cr[mf][j], ci[mf][j]);
          double2 v1 = v;
          if (a.mode == MODE_A_IMAG || a.mode == MODE_A_REAL) v1 = cscale(v, w);
          else if (a.mode == MODE_B_REAL) v1 = cconj(v);
          a.out[(int64_t)pl * nn + o] = v1;
          codes |= (uint32_t)(uint16_t)exponent_code(v1) << (16 * j);
          if (a.out2) {
            // the other imaginary-axis operand of the same G: v = G[r][c] goes to slot
            // (c, r) of the G^T layout (mode2 B) or, times w, to slot (r, c) of the G layout (mode2 A)
            int r, c;
            slot_rc(sa, a.mode, o, r, c);
            const bool tr = a.mode2 == MODE_B_IMAG;
            const int64_t i2 = (int64_t)pl * nn + sa.outinv[tr ? c * n + r : r * n + c];
            const double2 v2 = tr ? v : cscale(v, w);
            a.out2[i2] = v2;
            if (a.eout2) a.eout2[i2] = exponent_code(v2);
          }
        }
        if (a.eout && o0 < nn) *reinterpret_cast<uint32_t*>(a.eout + (int64_t)pl * nn + o0) = codes;
      }
    }
    __syncthreads();
  }
}

// --------------------------------------------------------------------------- LDOS from (U, lambda)
constexpr int kLdosE = 32;   // energies per CTA

// out[ie][r] += (eta / pi) sum_{k in this CTA's chunk} w_k sum_a |U[k][r][a]|^2 / ((e_ie - lambda_ka)^2 + eta^2),
// i.e. -Im G_rr(k, e + i eta) / pi summed over the chunk (atomicAdd into out)
__global__ void __launch_bounds__(256) spec_ldos_kernel(const double2* __restrict__ U, const double* __restrict__ lam,
                                                        const double* __restrict__ w, int64_t nk, int n,
                                                        const double* __restrict__ e, int n_e, double eta,
                                                        int64_t k_per_cta, double* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem[];
  double* P = reinterpret_cast<double*>(smem);   // [n][n] |U|^2
  double* L = P + n * n;                          // [kLdosE][n]
  double* acc = L + kLdosE * n;                   // [kLdosE][n]
  const int e0 = blockIdx.x * kLdosE;
  const int ne = min(kLdosE, n_e - e0);
  const int64_t k0 = (int64_t)blockIdx.y * k_per_cta, k1 = min(nk, k0 + k_per_cta);
  for (int o = threadIdx.x; o < kLdosE * n; o += blockDim.x) acc[o] = 0.0;
  for (int64_t k = k0; k < k1; ++k) {
    __syncthreads();
    const double2* Uk = U + k * (int64_t)n * n;
    for (int o = threadIdx.x; o < n * n; o += blockDim.x) {
      const double2 u = Uk[o];
      P[o] = u.x * u.x + u.y * u.y;
    }
    for (int o = threadIdx.x; o < ne * n; o += blockDim.x) {
      const double x = e[e0 + o / n] - lam[k * n + o % n];
      L[o] = 1.0 / (x * x + eta * eta);
    }
    __syncthreads();
    const double wk = w[k];
    for (int o = threadIdx.x; o < ne * n; o += blockDim.x) {
      const int ie = o / n, r = o % n;
      const double* pr = P + r * n;
      const double* le = L + ie * n;
      double s = 0.0;
      for (int a = 0; a < n; ++a) s = fma(pr[a], le[a], s);
      acc[o] = fma(wk, s, acc[o]);
    }
  }
  __syncthreads();
  const double f = eta / 3.141592653589793238462643383279502884;
  for (int o = threadIdx.x; o < ne * n; o += blockDim.x) atomicAdd(out + (int64_t)(e0 + o / n) * n + o % n, f * acc[o]);
}

// --------------------------------------------------------------------------- expectation sums from (U, lambda)
// For the occupations and moments only the orbital-diagonal spin blocks of G summed over
// the energies of each k are needed:
//   S(r, c) = sum_ie w(ie, k) G_rc(k, z_ie) = sum_a U[r][a] f_a conj(U[c][a]),
//   f_a = sum_ie w(ie, k) / (z_ie - lambda_a),  z_ie = zr + i (zi + y_ie),
// so each k costs n x n_e divisions and 4 n entries of n terms.  out: per-CTA slices of
// [n / 2 orbitals][uu, dd, ud, du] (rows[2 o], rows[2 o + 1] = up / down row of orbital o).
__global__ void __launch_bounds__(256) spec_expect_kernel(const double2* __restrict__ U, const double* __restrict__ lam,
                                                          int64_t nk, int n, const double* __restrict__ ylist,
                                                          int64_t n_e, const double* __restrict__ w, double zr,
                                                          double zi, const int* __restrict__ rows,
                                                          double2* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem[];
  double2* f = reinterpret_cast<double2*>(smem);   // [n]
  double2* acc = f + n;                            // [2 n]
  for (int e = threadIdx.x; e < 2 * n; e += blockDim.x) acc[e] = make_double2(0.0, 0.0);
  for (int64_t k = blockIdx.x; k < nk; k += gridDim.x) {
    __syncthreads();
    for (int a = threadIdx.x; a < n; a += blockDim.x) {
      const double l = lam[k * n + a];
      double fr = 0.0, fi = 0.0;
      const double x = zr - l;
      for (int64_t ie = 0; ie < n_e; ++ie) {
        const double y = zi + ylist[ie];
        const double inv = w[ie * nk + k] / (x * x + y * y);
        fr = fma(x, inv, fr);
        fi = fma(-y, inv, fi);
      }
      f[a] = make_double2(fr, fi);
    }
    __syncthreads();
    const double2* Uk = U + k * (int64_t)n * n;
    for (int e = threadIdx.x; e < 2 * n; e += blockDim.x) {
      const int o = e >> 2, q = e & 3;
      const int ru = rows[2 * o], rd = rows[2 * o + 1];
      const int r = (q == 0 || q == 2) ? ru : rd, c = (q == 0 || q == 3) ? ru : rd;
      double2 s = make_double2(0.0, 0.0);
      for (int a = 0; a < n; ++a) s = cfma(cmul(Uk[(int64_t)r * n + a], f[a]), cconj(Uk[(int64_t)c * n + a]), s);
      acc[e] = cadd(acc[e], s);
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 2 * n; e += blockDim.x) partial[(size_t)blockIdx.x * 2 * n + e] = acc[e];
}

}  // namespace

// --------------------------------------------------------------------------- host side
cudaError_t launch_spec_expect(const double2* U, const double* lam, int64_t nk, int n, const double* ylist, int64_t n_e,
                               const double* w, double zr, double zi, const int* rows, double2* partial, int grid,
                               cudaStream_t s) {
  if (nk <= 0) return cudaSuccess;
  const size_t smem = sizeof(double2) * 3 * (size_t)n;
  spec_expect_kernel<<<grid, 256, smem, s>>>(U, lam, nk, n, ylist, n_e, w, zr, zi, rows, partial);
  return cudaGetLastError();
}

cudaError_t launch_spec_ldos(const double2* U, const double* lam, const double* w, int64_t nk, int n,
                             const double* e, int n_e, double eta, double* out, int num_sms, cudaStream_t s) {
  if (nk <= 0 || n_e <= 0) return cudaSuccess;
  const size_t smem = sizeof(double) * ((size_t)n * n + 2 * (size_t)kLdosE * n);
  cudaError_t err = cudaFuncSetAttribute(spec_ldos_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  err = cudaMemsetAsync(out, 0, sizeof(double) * (size_t)n_e * n, s);
  if (err != cudaSuccess) return err;
  const int eb = (n_e + kLdosE - 1) / kLdosE;
  const int64_t kchunks = std::max<int64_t>(1, std::min<int64_t>(nk, (int64_t)4 * num_sms / eb));
  const int64_t kper = (nk + kchunks - 1) / kchunks;
  const dim3 grid((unsigned)eb, (unsigned)((nk + kper - 1) / kper));
  spec_ldos_kernel<<<grid, 256, smem, s>>>(U, lam, w, nk, n, e, n_e, eta, kper, out);
  return cudaGetLastError();
}

size_t eig_smem_bytes_form(int n, bool packed) {
  const size_t na = packed ? (size_t)n * (n + 1) / 2 : (size_t)n * n;
  return sizeof(double2) * (na + (size_t)n * n) + sizeof(Rot) * (size_t)(n / 2) + sizeof(double) * 32;
}

int eig_optin() {
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
  return optin;
}

// the full A when A and U both fit in shared memory, else the packed upper triangle
bool eig_packed(int n, int optin) { return eig_smem_bytes_form(n, false) > (size_t)optin; }

size_t eig_smem_bytes(int n) { return eig_smem_bytes_form(n, eig_packed(n, eig_optin())); }

// the unpacked kernel (A and U both in shared memory): fast enough to diagonalise per k even
// where few energies share a k list
int eig_fast(int n) {
  if (n % 2 != 0 || n < 2 || n > 32 * kEigCols) return 0;
  return !eig_packed(n, eig_optin());
}

int eig_supported(int n) {
  if (n % 2 != 0 || n < 2 || n > 32 * kEigCols) return 0;
  const int optin = eig_optin();
  return eig_smem_bytes_form(n, eig_packed(n, optin)) <= (size_t)optin;
}

cudaError_t launch_eig(const double2* H, int64_t nk, int n, double2* U, double* lam, int* status, int num_sms,
                       cudaStream_t s) {
  if (nk <= 0) return cudaSuccess;
  if (!eig_supported(n)) return cudaErrorInvalidValue;
  const bool packed = eig_packed(n, eig_optin());
  const size_t smem = eig_smem_bytes_form(n, packed);
  auto kernel = packed ? eig_jacobi_kernel<true> : eig_jacobi_kernel<false>;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kEigThreads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm <= 0) return cudaErrorInvalidValue;
  const int64_t grid = std::min<int64_t>(nk, (int64_t)num_sms * per_sm);
  kernel<<<(unsigned)grid, kEigThreads, smem, s>>>(H, nk, n, U, lam, status);
  return cudaGetLastError();
}

int spectral_supported(int mode, int mode2, bool has_out2) {
  const bool m = mode == MODE_RAW || mode == MODE_A_IMAG || mode == MODE_B_IMAG || mode == MODE_A_REAL ||
                 mode == MODE_B_REAL;
  if (!m) return 0;
  if (has_out2)
    return (mode == MODE_A_IMAG && mode2 == MODE_B_IMAG) || (mode == MODE_B_IMAG && mode2 == MODE_A_IMAG);
  return 1;
}

cudaError_t launch_green_spectral(const GreenArgs& g, const double2* U, const double* lam, const int* outinv,
                                  int num_sms, cudaStream_t s) {
  if (g.np <= 0) return cudaSuccess;
  if (g.n_e <= 0 || !U || !lam) return cudaErrorInvalidValue;
  if (!spectral_supported(g.mode, g.mode2, g.out2 != nullptr)) return cudaErrorInvalidValue;
  if (g.out2 && !outinv) return cudaErrorInvalidValue;
  if ((g.eout || g.eout2) && g.n % 2) return cudaErrorInvalidValue;   // paired 4-byte exponent stores
  SpecArgs sa;
  sa.g = g;
  sa.U = U;
  sa.lam = lam;
  sa.outinv = outinv;
  sa.kp = (g.n + 3) / 4 * 4;
  const size_t smem = spec_smem(g.n, sa.kp);
  const bool anti = g.mode == MODE_A_REAL;
  auto kernel = anti ? spec_green_kernel<true, kSpecThreads> : spec_green_kernel<false, kSpecThreads>;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kSpecThreads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm <= 0) return cudaErrorInvalidValue;
  int threads = kSpecThreads;
  if (per_sm == 1) {
    kernel = anti ? spec_green_kernel<true, 1024> : spec_green_kernel<false, 1024>;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 1024, smem);
    if (e != cudaSuccess) return e;
    if (per_sm <= 0) return cudaErrorInvalidValue;
    threads = 1024;
  }
  const int64_t ne = g.n_e;
  const int64_t ntask = ((g.p0 + g.np - 1) / ne - g.p0 / ne + 1) * ((ne + kSpecZ - 1) / kSpecZ);
  const int64_t grid = std::min<int64_t>(ntask, (int64_t)num_sms * per_sm);
  kernel<<<(unsigned)grid, threads, smem, s>>>(sa);
  return cudaGetLastError();
}

}  // namespace tg
