/*
 * titan_gpu.h -- C ABI of the B200 Green-function path (k-mesh x complex energy).
 *
 * Drop-in boundary for the reference's swappable Green-function routines.  A
 * Fortran host binds these with ISO_C_BINDING; every
 * array is caller-owned HOST memory in Fortran (column-major) order, complex
 * numbers are interleaved (re, im) doubles, and every call returns a status:
 *
 *     0            success
 *     > 0          singular (z - H(k)) at the returned 1-based point index
 *                  (the LAPACK info convention of invers, mod_tools.F90:814-827)
 *     TG_ERR_*     < 0, see below; tg_last_error() has the message
 *
 * One context per process and GPU; calls on one context are not re-entrant
 * (the reference calls these from the master thread only,
 * mod_mpi_pars.F90:49).
 */
#ifndef TITAN_GPU_H
#define TITAN_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TG_OK            0
#define TG_ERR_ARG      (-1)   /* bad argument (size, pointer, unsupported dimension) */
#define TG_ERR_CUDA     (-2)   /* CUDA runtime error */
#define TG_ERR_STATE    (-3)   /* call order: system / h0 / mesh not set */
#define TG_ERR_TIMEOUT  (-4)   /* a bounded device wait gave up */
#define TG_ERR_NOMEM    (-5)   /* device allocation failed */
#define TG_ERR_NUMERIC  (-6)   /* an iterative device solver did not converge */

/* Precision of the chi0 contraction (tg_chi0). */
#define TG_PREC_FP64     0     /* FP64 SIMT contraction */
#define TG_PREC_SPLIT    1     /* INT8-sliced tensor-core contraction (tcgen05), FP64 recombination */

typedef struct tg_ctx tg_ctx;

/* Context lifecycle.  Replaces create_handle / destroy_handle
 * (source/mod_cuda.F90:34,80; called at source/main.F90:81,431). */
int tg_create(int device, tg_ctx** ctx);
int tg_destroy(tg_ctx* ctx);
const char* tg_last_error(const tg_ctx* ctx);

/* Neighbour table of the tight-binding model: the data calchk reads
 * (source/mod_hamiltonian.F90:183-243; AtomTypes.F90:53-68).
 *   norb[n_atoms]                         orbitals per site
 *   cell_vec(3, n_neigh)                  Neighbors(k)%CellVector
 *   basis_idx(n_neigh)                    Neighbors(k)%BasisIndex (1-based)
 *   is_hopping(n_atoms, n_neigh)          Neighbors(k)%isHopping(i) (0/1)
 *   t0i(norb_max, norb_max, n_atoms, n_neigh) complex: Neighbors(k)%t0i(:,:,i)
 */
int tg_set_system(tg_ctx* ctx, int n_atoms, const int* norb, int norb_max, int n_neigh,
                  const double* cell_vec, const int* basis_idx, const int* is_hopping,
                  const double* t0i);

/* Local Hamiltonian h0(dimH, dimH) complex (mod_hamiltonian.F90:35-87, the
 * module array h0 that green() adds).  Set again whenever hee changes. */
int tg_set_h0(tg_ctx* ctx, int dimH, const double* h0);

/* Imaginary-axis (E, k) list: the flattened E_k_imag_mesh of
 * adaptiveMesh.F90:76-161 with y(E), bzs(E)%kp and wght(E)*bzs(E)%w per point. */
int tg_set_imag_mesh(tg_ctx* ctx, int64_t n_points, const double* y, const double* kp,
                     const double* w);

/* Real-axis BZ (realBZ%kp(3, nk), realBZ%w(nk), mod_BrillouinZone.F90:64-110). */
int tg_set_real_mesh(tg_ctx* ctx, int64_t n_k, const double* kp, const double* w);

/* chi0_HF(q, e): replaces eintshechi(q, e) (source/eintshechi.F90:2-178).
 *   (x2, p2)[n_real]   real-axis points of generate_real_epoints(e) (ignored when |e| < 1e-15)
 *   chiorb_hf(dimens, dimens) complex, the module array of mod_susceptibilities,
 *   already divided by 2 pi (eintshechi.F90:174).  precision: TG_PREC_*. */
int tg_chi0(tg_ctx* ctx, const double* q, double e, double Ef, double eta, double etap,
            int n_real, const double* x2, const double* p2, int precision, int dimens,
            double* chiorb_hf);

/* Batched chi0 over n_omega frequencies at one q: the imaginary-axis G(k, Ef+iy)
 * is computed once and reused for every frequency (it does not depend on e).
 *   e[n_omega]; x2, p2: (n_real, n_omega), column w = real-axis points of e[w];
 *   chiorb_hf(dimens, dimens, n_omega). */
int tg_chi0_batch(tg_ctx* ctx, const double* q, int n_omega, const double* e, double Ef,
                  double eta, double etap, int n_real, const double* x2, const double* p2,
                  int precision, int dimens, double* chiorb_hf);

/* Autotuning of the chi0 contraction schedule (on by default): the first call for each
 * contraction layout (precision, site-pair tiles, points per pass, chi dimension) times the
 * K-range split counts 1, 2, 4, ..., 64 of its contraction kernel on one pass with CUDA
 * events and keeps the fastest for the context's later calls; off uses the cost model
 * alone (and forgets the measured choices).  tg_tuning reports the split counts of the
 * last FP64 and split-precision calls.  No counterpart in the reference. */
int tg_set_autotune(tg_ctx* ctx, int enable);
int tg_tuning(const tg_ctx* ctx, int* nsplit_fp64, int* nsplit_split);

/* Error bound of the last tg_chi0 / tg_chi0_batch / tg_chi0_qbatch call (the err_est output
 * of the chi0 boundary): bound[r] for each of its n results (n = n_omega, or n_omega * n_q,
 * in the order of chiorb_hf) bounds ||chi_split - chi||_F / ||chi_split||_F, chi being the same
 * sums in exact arithmetic, from the split format alone: each operand element rounded to
 * 46 bits of its chunk's power-of-two scale, and the digit products the format drops.  A
 * worst-case bound, accumulated per chunk and site pair on the device.  0 for TG_PREC_FP64
 * results (the FP64 rounding that both paths share is not part of it); NaN after a call that
 * failed.  n other than the last call's result count is TG_ERR_ARG.  No counterpart in the
 * reference. */
int tg_chi0_error_bound(tg_ctx* ctx, int n, double* bound);

/* Points per chunk of the split-precision contraction (TG_PREC_SPLIT): each energy's
 * points are cut into chunks of at most this many, and every operand element gets one
 * power-of-two scale per chunk, so shorter chunks follow the magnitude of G along the k
 * list (more accurate near the real axis) at the cost of more accumulator drains.
 * 1 .. 16384; 0 restores the default (1024).  No counterpart in the reference. */
int tg_set_split_chunk(tg_ctx* ctx, int points);

/* chi0 for n_q wave vectors q(3, n_q) and n_omega frequencies (the loops of calculate_chi
 * over q and e, calculate_chi.F90:61-73, around eintshechi):
 *   chiorb_hf(dimens, dimens, n_omega, n_q), x2 / p2 as in tg_chi0_batch.
 * G2 = G(k, z) does not depend on q: when the imaginary axis is not a tabulated uniform
 * mesh (adaptive meshes, or H(k) tables above 8 GiB) every pass inverts and quantises it
 * once and contracts it with G1(k + q, z + e) of every (q, e).  The real axis then uses
 * spectral Green functions where the method and dimension allow (eigendecompositions of
 * H(k) once and of H(k + q) once per q, for every frequency; G2 formed again per q), or
 * beyond dimH 72 Householder tridiagonalisations of H(k) and of every H(k + q) (up to 8
 * nonzero q at once, memory permitting) with G2 formed once per pass and frequency for all
 * q, else one inversion of G2 per pass and frequency shared by the q.  On tabulated meshes the q run one after another,
 * each sharing G2 over its frequencies.  No counterpart in the reference. */
int tg_chi0_qbatch(tg_ctx* ctx, int n_q, const double* q, int n_omega, const double* e, double Ef,
                   double eta, double etap, int n_real, const double* x2, const double* p2,
                   int precision, int dimens, double* chiorb_hf);

/* Restricts chi0 (tg_chi0, tg_chi0_batch) to a subset of each site's orbitals:
 * mask(norb_max, n_atoms) flags the orbitals mu (both spins) that enter chi; null
 * restores every orbital (the reference's dimens = 4 sum_i nOrb_i^2).  With a mask,
 * dimens = 4 sum_i nc_i^2 (nc_i flagged orbitals of site i) and chiorb_hf is the
 * sub-block of the reference's chiorb_hf over those orbitals, in the same
 * sigmaimunu2i order restricted to them (sigma fastest, then nu, mu, site;
 * mod_System.F90:176-187).  Flagging the d orbitals gives the d-only chi whose RPA
 * Dyson solve (tg_dyson with U restricted to the same rows) equals the d-d block of
 * the full one, because U is non-zero only between d orbitals
 * (mod_susceptibilities.F90:106-159).  tg_set_system clears the mask.  No
 * counterpart in the reference. */
int tg_set_chi_orbitals(tg_ctx* ctx, const int* mask);

/* Occupations and moments: replaces expectation_values_greenfunction
 * (source/mod_expectation.F90:28-149).  All outputs (norb_max, n_atoms). */
int tg_expectation(tg_ctx* ctx, double Ef, double eta, double* rho, double* mx, double* my,
                   double* mz, double* mp);

/* tg_expectation without device allocation, for callers that cannot let a
 * library call allocate: a host that gives the GPU's memory to its own pool or
 * to another solver up front and budgets every byte of HBM itself.  No
 * counterpart in the reference.  Same outputs as tg_expectation under its
 * default method; this call always inverts per (k, z) point (Gauss-Jordan),
 * whatever tg_set_green_method chose.  H(k) is summed inside the kernel and the
 * partial sums live in a fixed 8 MiB device array of the library:
 * (16 x SMs + 1) x 2 dimH complex must fit (dimH <= 90 on a B200), else
 * TG_ERR_ARG before any work.  The first call on a context looks the array's
 * address up on the context's device (make it before any stream capture);
 * nothing has to start at zero; calls that overlap in time on one device race
 * on the shared array. */
int tg_expectation_noalloc(tg_ctx* ctx, double Ef, double eta, double* rho, double* mx, double* my,
                           double* mz, double* mp);

/* Orbital-diagonal GG tensor for the Jacobian and its adjoint:
 *   T(16, ncol, nrow, n_atoms(j), n_atoms(i)) complex with
 *   T[s',t,t',s; i,g; j,h] = sum_p w_p sum_{mu in g} sum_{nu in h}
 *        G(i s' mu, j t nu) G(j t' nu, i s mu),  G at Ef + i(y_p + eta),
 *   spin index order s' + 2 t + 4 t' + 8 s (0 = up).
 * Row groups of site i: d orbitals one by one, then all non-d orbitals summed
 * (nrow = nd + 1); column groups: d orbitals one by one (ncol = nd) when
 * orbital_resolved != 0; dmask(norb_max, n_atoms) flags the d orbitals
 * (Types%dOrbs) and may be null otherwise.  With orbital_resolved == 0 every site has one row
 * group and one column group holding all its orbitals (the (V, B) adjoint).
 * This is the contraction inside calcJacobian_greenfunction
 * (mod_self_consistency.F90:843-1127); the host maps it onto the Jacobian. */
int tg_gg_tensor(tg_ctx* ctx, double Ef, double eta, int orbital_resolved, const int* dmask, double* T);

/* Fermi-level column of calcJacobian_greenfunction (mod_self_consistency.F90:1131-1196):
 *   D(4, norb_max, n_atoms) complex: sum_k w_k tr_spin[sigma_a G_ii(mu,mu)](Ef + i eta)
 *   over realBZ, sigma_a = (1, x, y, z). */
int tg_fermi_column(tg_ctx* ctx, double Ef, double eta, double* D);

/* Jacobian of the self-consistency equations: replaces
 * calcJacobian_greenfunction(jacobian, N) (source/mod_self_consistency.F90:795-1205).
 * Unknowns per site i (set_hamiltonian_variables, :1754-1780): the occupation of each
 * d orbital when Un(i) != 0, then (mx, my, mz) of the d shell when Um(i) != 0, and
 * E_F last unless fixEf.  dmask(norb_max, n_atoms) flags the d orbitals (Types%dOrbs),
 * Un/Um(n_atoms) the Hubbard parameters; jac(neq, neq) column-major real.
 * J = (1/pi) sum_{k,E} w Re Tr_d[sigma_a G_ij M_b G_ji] (+ the E_F column from the
 * real-axis BZ at E_F + i eta) minus the identity on the first neq - 1 entries. */
int tg_jacobian(tg_ctx* ctx, double Ef, double eta, const int* dmask, const double* Un,
                const double* Um, int fixEf, int neq, double* jac);

/* Number of unknowns (the N of calcJacobian_greenfunction) and, when per is not
 * null, the first unknown of each site: per(n_atoms + 1).  Host only. */
int tg_jacobian_layout(int n_atoms, const int* norb, int norb_max, const int* dmask,
                       const double* Un, const double* Um, int fixEf, int* per);

/* Host-only assembly of the Jacobian from the GG tensor T (tg_gg_tensor with
 * orbital_resolved = 1, shape (16, ncol, nrow, n_atoms, n_atoms)) and the
 * Fermi column D (tg_fermi_column; ignored when fixEf).  No GPU work. */
int tg_jacobian_assemble(int n_atoms, const int* norb, int norb_max, const int* dmask,
                         const double* Un, const double* Um, int fixEf, int nrow, int ncol,
                         const double* T, const double* D, int neq, double* jac);

/* Adjoint of the site occupations and moments with respect to an on-site
 * potential V_i and exchange field B_i added to every orbital of site i,
 * h0 -> h0 + sum_i P_i (V_i sigma_0 + B_i . sigma).  A(4 n_atoms, 4 n_atoms) column-major,
 * A(a + 4 i, b + 4 j) = d x_{i,a} / d p_{j,b} with x = (n, mx, my, mz) of
 * expectation_values_greenfunction (mod_expectation.F90:28-149) summed over the
 * site's orbitals and p = (V, Bx, By, Bz): (1/pi) sum w Re Tr[P_i sigma_a G P_j sigma_b G].
 * No counterpart in the reference (its Jacobian uses the d-shell variables above). */
int tg_adjoint_vb(tg_ctx* ctx, double Ef, double eta, double* A);

/* tg_adjoint_vb with the potential and the field acting on a subset of each site's
 * orbitals and the observables summed over the same subset: mask(norb_max, n_atoms)
 * flags the orbitals (null = every orbital, i.e. tg_adjoint_vb).  With the d orbitals
 * flagged, p = (V, B) is the d-shell field of update_Umatrix (mod_U_matrix.F90:29-55),
 * whose exchange part is B_i = -(Um_i / 2) m_i on the d orbitals, so with Un = 0 the
 * reference's moment Jacobian is J + 1 = -(Um / 2) A on the moment rows and columns.
 * No counterpart in the reference. */
int tg_adjoint_vb_orbitals(tg_ctx* ctx, double Ef, double eta, const int* mask, double* A);

/* n_atoms, norb_max and (when norb is not null) norb(n_atoms) of the system set by
 * tg_set_system. */
int tg_system_shape(const tg_ctx* ctx, int* n_atoms, int* norb_max, int* norb);

/* RPA Dyson solve chi = (1 + chi_hf U)^-1 chi_hf in FP64 on the GPU
 * (calculate_chi.F90:85-89).  All matrices (dimens, dimens) complex. */
int tg_dyson(tg_ctx* ctx, int dimens, const double* chi_hf, const double* umat, double* chi);

/* Disturbance response to an electric field: replaces eintshe(q, e)
 * (source/eintshe.F90:2-309) for one frequency e.
 *   tchi(dimens, 4) complex = prefactor . (1/2pi) sum_{k,E} w df1iikl(k, E)
 * with df1iikl the vertex sandwich of G(k + q, E + e), dtdk(k) (dtdksub.F90:2-28,
 * efield(3) the unit field vector u of ElectricFieldVector) and G(k, E) on the
 * diagonal site blocks, summed over the imaginary-axis mesh of tg_set_imag_mesh and,
 * when |e| >= 1e-15, over n_real real-axis energies x2/p2 (generate_real_epoints)
 * times the real-axis BZ of tg_set_real_mesh.  prefactor(dimens, dimens) complex is
 * the reference's (1 + chi_hf U)^-1 (calculate_all.F90:117-120); null = identity,
 * which returns the bare integral.  Row order of tchi: sigmaimunu2i. */
int tg_she(tg_ctx* ctx, const double* q, double e, double Ef, double eta, double etap, int n_real,
           const double* x2, const double* p2, const double* efield, const double* prefactor,
           int dimens, double* tchi);

/* Linear-SOC susceptibility: replaces eintshechilinearsoc(q, e) (source/eintshechi.F90:182-414).
 * The context's h0 (tg_set_h0) must be the Hamiltonian without the local spin-orbit blocks
 * and vsoc(dimH, dimH) complex those blocks (the hk / vsoc split of hamiltklinearsoc,
 * mod_hamiltonian.F90:304-396).  With G0 = (z - h0 - H(k))^-1:
 *   chiorb_hf(dimens, dimens)   chi0_HF of G0 (as tg_chi0 with that h0),
 *   chiorb_lsoc(dimens, dimens) chi(G0 V G0 (k+q, E+e), G0(k, E)) + chi(G0(k+q, E+e), G0 V G0 (k, E)),
 * both divided by 2 pi.  The real-axis part runs over all n_real energies (the reference's
 * loop stops after the first energy's k points, eintshechi.F90:321).  FP64, Gauss-Jordan per
 * point; dimH up to 68 (3 dimH^2 complex of shared memory). */
int tg_chi0_linear_soc(tg_ctx* ctx, const double* q, double e, double Ef, double eta, double etap,
                       int n_real, const double* x2, const double* p2, const double* vsoc, int dimens,
                       double* chiorb_hf, double* chiorb_lsoc);

/* Exchange coupling J_ij(q): replaces jij_energy(q, Jij) (source/jij_energy.F90:6-242) in
 * the normal state.  With dBxc/dm = -Um_i/2 (sigma^d_mu - (sigma^d . e_i) e_{i mu}) on the d
 * orbitals (dmask(norb_max, n_atoms), the d-moment directions evec(3, n_atoms), Um(n_atoms)):
 *   J(i, j, mu, nu) = -1/(2 pi) sum_{k,E} w [Tr(A^i_mu G_ij(k) A^j_nu G_ji(k-q))
 *                                           + conj Tr(A^i_mu G_ij(k-q) A^j_nu G_ji(k))]
 * over the imaginary-axis mesh at Ef + i(y + eta); J(n_atoms, n_atoms, 3, 3) complex.
 * Gauss-Jordan per point (two inversions: k and k - q). */
int tg_jij(tg_ctx* ctx, const double* q, double Ef, double eta, const double* evec, const double* Um,
           const int* dmask, double* J);

/* Orbital-resolved on-site spin density of the sum rule: replaces calcSmunu
 * (source/mod_sumrule.F90:162-245).  With A = sum_{k,E} w G(i, i) over the imaginary-axis
 * mesh at Ef + i(y + eta) and imgXY(mu, nu) = (A(nu X, mu Y) + conj A(mu Y, nu X)) / 2 pi
 * (+ 1/2 on the uu and dd diagonals):
 *   S(mu, nu, 1, i) = imgud + imgdu,  S(:, :, 2, i) = i (imgud - imgdu),  S(:, :, 3, i) = imguu - imgdd,
 * S(norb_max, norb_max, 3, n_atoms) complex (Smunuiivec).  Gauss-Jordan per point. */
int tg_smunu(tg_ctx* ctx, double Ef, double eta, double* S);

/* Ground-state orbital density of every site: the Green-function integral of
 * calc_GS_L_and_E_greenfunction (source/mod_expectation.F90:912-982),
 *   gupgd(nu, mu, i) = (1/pi) sum_{k,E} w (G(i mu up, i nu up) + G(i mu dn, i nu dn))
 * at Ef + i(y + eta) over the imaginary-axis mesh; gupgd(norb_max, norb_max, n_atoms)
 * complex.  The orbital moments follow on the host as in calculate_L (:984-1009):
 * lxm(i) = Re sum_{mu,nu} lvec(mu, nu, 1) gupgd(mu, nu, i), and likewise lym, lzm and the
 * local-frame lxpm.. with lpvec.  The band energy is not computed (the reference sets it
 * to zero on this path).  Gauss-Jordan per point. */
int tg_gs_orbital(tg_ctx* ctx, double Ef, double eta, double* gupgd);

/* Local density of states on the real axis: replaces ldos_energy(e, ldosu, ldosd)
 * (source/mod_LDOS.F90:95-150) for n_e energies at once:
 *   ldosu(mu, i, ie) = -(1/pi) sum_k w_k Im G(i up mu, i up mu; k, e(ie) + i eta)
 * (ldosd with the down block) over the real-axis BZ of tg_set_real_mesh;
 * ldosu, ldosd(norb_max, n_atoms, n_e).  With TG_GREEN_AUTO / TG_GREEN_SPECTRAL each
 * H(k) is diagonalised once for all energies; TG_GREEN_GAUSS_JORDAN inverts per (k, e). */
int tg_ldos(tg_ctx* ctx, int n_e, const double* e, double eta, double* ldosu, double* ldosd);

/* How G(k, z) is computed.  Spectral: on meshes where every energy uses the same
 * k list (uniform imaginary axis, the real-axis BZ) H(k) is diagonalised once per k
 * (Jacobi, FP64) and G(k, z) = U diag(1/(z - lambda)) U^+ is formed for all energies
 * with FP64 tensor-core GEMMs.  Gauss-Jordan: one inversion per (k, z), the
 * reference's invers (mod_tools.F90:796-829).  Near the real axis the spectral G
 * carries errors up to eps |H| / Im z relative (1e-13 at Im z = 1e-3): the mixing of
 * nearly degenerate eigenvectors times the difference of their weights, while the
 * inversion stays near eps.  Sums over the mesh average this out for chi0 (same
 * error against the FP64 oracle as Gauss-Jordan), but the disturbance integral feeds
 * B_eff through an ill-conditioned site-reduced chi^-1, and the occupations feed a Newton
 * iteration whose step tolerance (mag_tol = 1e-12) the spectral noise exceeds, so:
 *   TG_GREEN_AUTO (default)  spectral for chi0 (dimH <= 72) and tg_ldos; for chi0 beyond
 *                            dimH 72, G over the rows chi needs from one Householder
 *                            tridiagonalisation per k, H = Q T Q^H, and per energy
 *                            Q_S (z - T)^-1 Q_S^H (LU-like accuracy); Gauss-Jordan for
 *                            tg_expectation; for tg_she spectral at Im z >= 10 eta and
 *                            Gauss-Jordan below and on the real axis (dimH 36; elsewhere
 *                            Gauss-Jordan)
 *   TG_GREEN_GAUSS_JORDAN    Gauss-Jordan everywhere
 *   TG_GREEN_SPECTRAL        spectral wherever the mesh allows (tg_she ~4x faster,
 *                            tg_expectation one eigendecomposition per k for all energies)
 * The eigendecomposition handles even dimH up to 96 and the tridiagonalisation any dimH up
 * to 288; meshes whose energies do not share a k list (adaptive imaginary axes) always use
 * Gauss-Jordan there.  No counterpart in the reference. */
#define TG_GREEN_AUTO          0
#define TG_GREEN_GAUSS_JORDAN  1
#define TG_GREEN_SPECTRAL      2
int tg_set_green_method(tg_ctx* ctx, int method);

/* Test hook: eigenvalues lam(dimH, nk) and eigenvectors of h0 + H(k) from the Jacobi
 * kernel behind TG_GREEN_AUTO, U(dimH, dimH, nk) with U(a, :, k) = eigenvector a (the
 * device's row-major [k][r][a] layout); TG_ERR_NUMERIC if a matrix did not converge in
 * 30 sweeps. */
int tg_eig_batch(tg_ctx* ctx, int64_t nk, const double* kp, double* lam, double* U);

/* Test hooks.  G(dimH, dimH, nz) = (z - h0 - H(k))^-1 for nz (k, z) pairs,
 * and H(dimH, dimH, nk) = h0 + calchk(k). */
int tg_green_batch(tg_ctx* ctx, int64_t nz, const double* z, const double* kp, double* G);
int tg_hamiltk_batch(tg_ctx* ctx, int64_t nk, const double* kp, double* H);

/* Measured FP64 throughput of the current device (TFLOP/s): a DFMA loop (8 independent
 * chains per thread) and a DMMA loop (mma.sync.m8n8k4.f64, 4 chains per warp), 4 CTAs of
 * 256 threads per SM, timed with CUDA events.  The denominators of the inversion
 * kernels' roofline.  ctx may be null.  No counterpart in the reference. */
int tg_fp64_peak(tg_ctx* ctx, double* tflops_dfma, double* tflops_dmma);

/* Test hook: r[i] = the pivot reciprocal of the Gauss-Jordan kernels applied to s[i] > 0
 * (the hardware approximation refined by three Newton-Raphson steps). */
int tg_rcp_check(int64_t n, const double* s, double* r);

/* Device timing of the last tg_chi0/tg_chi0_batch call (CUDA events on the
 * context's stream): ms[0] imaginary-axis G2 inversions, ms[1] contraction and
 * the other inversions, ms[2] epilogue, ms[3] whole call; when per-launch
 * profiling is on (tg_profile), ms[4..9] = (total ms, timed regions) of the
 * inversion, contraction and epilogue kernels, ms[11..12] the same for the
 * split-precision quantisation (row maxima + digit planes); ms[10] = kernels
 * launched.  ms must hold 13 doubles. */
int tg_last_timing(const tg_ctx* ctx, double* ms);
int tg_profile(tg_ctx* ctx, int enable);

#ifdef __cplusplus
}
#endif
#endif /* TITAN_GPU_H */
