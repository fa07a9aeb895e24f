/* scatt_b200.h -- C ABI of the B200 static-exchange scattering library.
 *
 * Drop-in boundary for the per-energy hot path of static-exchangeHF
 * (SchurInverter -> ForwardRPropagator -> KMatrixExtractor ->
 *  BackPropagator -> AsymptoticAmplitudes -> DipoleMatrixElement).
 *
 * Conventions
 *   - every function returns an int status (SCATT_OK = 0); the message of
 *     the last failure on the calling thread is scatt_last_error();
 *   - no exceptions cross this boundary; no C++ or torch types appear in it;
 *   - matrices are FP64, column-major, with explicit leading dimensions
 *     (Eigen's default layout, as in src/scatt/GpuPropagate.hpp:188-193);
 *   - all host arrays are caller-owned; the library owns device memory;
 *   - there is no CPU fallback: without a CUDA device every compute entry
 *     point returns SCATT_ERR_NO_DEVICE.
 */
#ifndef SCATT_B200_H
#define SCATT_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define SCATT_OK                 0
#define SCATT_ERR_ARG            1   /* bad argument / shape                        */
#define SCATT_ERR_CUDA           2   /* CUDA runtime error                          */
#define SCATT_ERR_SIZE           3   /* size beyond a kernel limit                  */
#define SCATT_ERR_SINGULAR       4   /* zero pivot (LapackInverse.hpp:73-86 throws)  */
#define SCATT_ERR_NONFINITE      5   /* NaN / Inf pivot                             */
#define SCATT_ERR_CLOSED_CHANNEL 6   /* AsymptoticAmplitudes.cpp:177-186 abort      */
#define SCATT_ERR_NO_DEVICE      7   /* no CUDA device visible                      */
#define SCATT_ERR_STATE          8   /* call order (e.g. solve before upload)       */
#define SCATT_ERR_OOM            9   /* device allocation failed                    */
#define SCATT_ERR_FIT_WINDOW    10   /* AsymptoticAmplitudes.cpp:85-91 abort        */
#define SCATT_ERR_IO            11   /* file missing, unreadable or not the expected HDF5 */

/* ------------------------------------------------------------------ misc */
const char* scatt_version(void);
const char* scatt_last_error(void);
/* Number of visible CUDA devices (0 without a GPU; never fails on a CPU host). */
int scatt_device_count(int* count);

/* ------------------------------------------------------- angular algebra
 * Host-side precompute shared with the device tables.
 * Replace src/angular/Gaunt.hpp:65-135 (gaunt_real over GSL 3j) and
 * src/scatt/DipoleMatrixElement.cpp:80-95 (angular_dipole, velocity_coef). */
double scatt_wigner3j(int j1, int j2, int j3, int m1, int m2, int m3);
double scatt_gaunt_real(int l1, int m1, int l2, int m2, int l3, int m3);
double scatt_angular_dipole(int l_mu, int m_mu, int q, int l_nu, int m_nu);
double scatt_velocity_coef(int l_mu, int l_nu);
/* Riccati-Bessel x j_l(x) and Riccati-Neumann x y_l(x) (the same routine the
 * kernels use).  Replace the GSL calls of ForwardRPropagator.cpp:64-75,
 * KMatrixExtractor.cpp:50-73, AsymptoticAmplitudes.cpp:39-62. */
double scatt_riccati_j(int l, double x);
double scatt_riccati_y(int l, double x);

/* ------------------------------------------------ dense device building blocks
 * Batched inverse of `count` n x n matrices (contiguous, ld = n) with partial
 * pivoting; symmetrize != 0 returns 0.5 (X + X^T).  status (may be NULL)
 * receives 2 ints per matrix: device status code, first failing column.
 * Orders up to 8192 under the automatic and row-contiguous schemes (above
 * 1280 the panels run on a thread-block cluster of up to 8 CTAs per
 * matrix); larger orders return SCATT_ERR_SIZE.
 * Replaces inverse_general / inverse_symmetric_indefinite
 * (src/scatt/LapackInverse.hpp:53-178). */
int scatt_inverse_batched(int n, int count, const double* A, double* out,
                          int symmetrize, int* status);

/* scatt_inverse_batched without device allocation, for callers that cannot
 * call cudaMalloc: a host whose own allocator already holds the device's free
 * memory (a framework's caching allocator, a fixed per-rank budget), or a
 * latency-bound caller that cannot accept the device-wide synchronisation of
 * cudaMalloc / cudaFree.  Every device buffer (matrix copies, ping-pong
 * buffers, pivot maps, panel windows, status words, entry table) is carved
 * from one static 64 MiB device array.  The array is reserved on a device
 * when the library's module holding it loads there -- at the first use of
 * this entry point under CUDA's default lazy module loading, at context
 * creation under CUDA_MODULE_LOADING=EAGER -- and is held until the process
 * exits.
 * Limits: n <= 1280, count <= 256, and
 * 8 count (3 n^2 + 128 n) + 4 count (4 n + 2) + 80 count bytes (each of
 * the nine pieces rounded up to 256) <= 64 MiB; larger requests return SCATT_ERR_SIZE before
 * any device work.  The first call on a device resolves the array's address
 * (cudaGetSymbolAddress) and creates the non-blocking stream the calls run
 * on; it should come before any stream capture.  Calls do not synchronise
 * with the caller's other streams, but return only after their host copies.
 * Calls that overlap in time on one device (several host threads) share the
 * array and race.  No counterpart in the reference. */
int scatt_inverse_batched_noalloc(int n, int count, const double* A, double* out,
                                  int symmetrize, int* status);

/* C = alpha op(A) op(B) + beta C on the device, host buffers (op: 0 = N, 1 = T). */
int scatt_dgemm(int opA, int opB, int M, int N, int K, double alpha,
                const double* A, int lda, const double* B, int ldb,
                double beta, double* C, int ldc);

/* Device-resident timing of scatt_inverse_batched's kernels on seeded
 * matrices (CUDA events around the kernels only); used by the inverse
 * benchmark (python -m scatt_b200.inverse_bench). */
int scatt_bench_inverse(int n, int count, int reps, double* ms_per_call);
/* Device-resident timing of one batched GEMM call (count products
 * C = op(A) op(B), M x N x K, seeded operands; sym != 0 computes the lower
 * triangle and mirrors it, M == N) by CUDA events around the call, mean of
 * reps calls after one untimed call; used by the GEMM benchmark
 * (python -m scatt_b200.gemm_bench).  No counterpart in the reference. */
int scatt_bench_gemm(int opA, int opB, int M, int N, int K, int count, int sym, int reps,
                     double* ms_per_call);
/* Blocking scheme of every dense inverse (the entry points and the solver):
 * 0 = automatic (default): scheme 3 above order 512, scheme 2 below,
 * 1 = single-level (rank-16 updates, row pivoting),
 * 2 = two-level column-major (64-column windows, row pivoting),
 * 3 = two-level on the row-contiguous view of the buffer (pivots by columns
 *     of A, which for a symmetric A is the row-pivoting sequence),
 * 4 = scheme 3 with 128-column outer windows (rank-128 trailing updates;
 *     the allocation-free entry point keeps 64-column windows),
 * 5, 6 = schemes 3 and 4 with the small cluster panel (clusters of
 *     384-row CTAs, small enough to share an SM with the trailing update).
 * All give the same inverse up to rounding.  The setting is process-wide and
 * applies from the next inverse on, also in solves running on other threads. */
int scatt_set_inverse_blocking(int scheme);

/* Autotuner of the two-level inverses: times scheme 2 and scheme 3 (the
 * latter with and without look-ahead, and with 64- and 128-column windows)
 * with every panel shape that holds order n, on a batch of `count` seeded
 * matrices of order n (reps timed calls each), and keeps the fastest for
 * (current device, n, count).  Under the automatic scheme
 * (scatt_set_inverse_blocking(0)) every later inverse of exactly that order
 * and batch on that device -- the solver's Schur and R^-1 batches included
 * -- uses the kept choice.  Outputs (each may be NULL): the scheme (2 or 3),
 * the panel shape (0..4: 1x8, 2x8, 3x8, 3x12, 5x8 rows per thread x warps;
 * 5: the cluster panel of orders above 1280; 6: the small cluster panel,
 * row-contiguous scheme, orders up to 3072), look-ahead (0/1), the window
 * width (64 or 128) and the chosen configuration's milliseconds per call.
 * Orders 1..8192 (above 1280 only scheme 3 runs).  No counterpart in the
 * reference. */
int scatt_autotune_inverse(int n, int count, int reps, int* scheme, int* panel, int* look_ahead,
                           int* window, double* best_ms);

/* ------------------------------------------- per-step compatibility seam
 * The reference's per-radial-step device interface (GpuForwardStepper,
 * GpuSinvStepper, GpuBackStepper in src/scatt/GpuPropagate.hpp:83-279),
 * kept for callers and checks written against it.  Each stepper keeps its
 * carried state on the device and takes one step's operands as host
 * buffers (column-major FP64); the batched solver does not use them.
 * max_asym_out (may be NULL) receives max |X - X^T| of the result. */
typedef struct scatt_fwd_stepper scatt_fwd_stepper;
typedef struct scatt_sinv_stepper scatt_sinv_stepper;
typedef struct scatt_back_stepper scatt_back_stepper;

/* Rinv_n = sym((12 W_inv - 10 I - Rinv_{n-1})^-1); Rinv_{n-1} starts at 0
 * or at the matrix given to scatt_fwd_stepper_init. */
int scatt_fwd_stepper_create(int device, int n_total, scatt_fwd_stepper** out);
int scatt_fwd_stepper_destroy(scatt_fwd_stepper* h);
int scatt_fwd_stepper_init(scatt_fwd_stepper* h, const double* rprev_inv);
int scatt_fwd_stepper_step(scatt_fwd_stepper* h, const double* w_inv, double* rinv_out,
                           double* max_asym_out);
/* Sinv = sym((A - B diag(Dinv) B^T)^-1); B = Dinv = NULL gives sym(A^-1)
 * (GpuSinvStepper::step_inverse_only). */
int scatt_sinv_stepper_create(int device, int n_psi, int n_f, scatt_sinv_stepper** out);
int scatt_sinv_stepper_destroy(scatt_sinv_stepper* h);
int scatt_sinv_stepper_step(scatt_sinv_stepper* h, const double* A, const double* B,
                            const double* dinv, double* sinv_out, double* max_asym_out);
/* Z <- Rinv Z; Y = W_inv Z; psi = first n_psi rows of Y (n_psi x n_psi),
 * f = the rest (n_f x n_psi, may be NULL). */
int scatt_back_stepper_create(int device, int n_total, int n_psi, scatt_back_stepper** out);
int scatt_back_stepper_destroy(scatt_back_stepper* h);
int scatt_back_stepper_init(scatt_back_stepper* h, const double* Z);
int scatt_back_stepper_step(scatt_back_stepper* h, const double* rinv, const double* w_inv,
                            double* psi_out, double* f_out);
int scatt_back_stepper_get_z(scatt_back_stepper* h, double* Z_out);

/* ------------------------------------------------------ per-scan solver
 * The reference runs one energy at a time through run_one_energy
 * (src/main.cpp:1081-1623); here a batch of energies is solved together,
 * lock-step over the radial grid, with every intermediate (Sinv, R^-1, the
 * dipole sweeps) resident in HBM.  Stage order and policies follow the
 * reference classes (SchurInverter, ForwardRPropagator, KMatrixExtractor,
 * BackPropagator, AsymptoticAmplitudes, DipoleMatrixElement). */
typedef struct scatt_ctx scatt_ctx;

/* Energy-independent inputs of one scan: the content of the preprocessing
 * file the reference reads (src/io/HDF5Reader.hpp:42-86). */
typedef struct {
    int    Nr;            /* radial points (SolverParams::n_grid)                        */
    double dr;            /* step; the preprocessing grid is r = ir * dr                 */
    int    l_cont_max;    /* largest continuum l of any energy in the scan               */
    int    n_occ;         /* occupied orbitals in the exchange sum and orthogonalisation */
    int    n_orb;         /* orbitals stored in psi_lm (>= n_occ)                        */
    int    Nlm_store;     /* angular channels stored per orbital                         */
    int    Nr_store;      /* radial points stored per orbital (<= Nr)                    */
    const double* psi_lm; /* [n_orb][Nlm_store][Nr_store] C order: F_{i,lambda}(ir dr)    */
    int    init_state;    /* orbital used as dipole initial state; -1 = n_occ - 1 (HOMO)  */
    int    n_H;           /* rows of V_H supplied                                        */
    const double* V_H;    /* [n_H][Nr] C order: Hartree multipoles V_H,sigma(ir dr)       */
    int    n_atoms;
    const double* atoms;  /* [n_atoms][4]: Z, x, y, z (bohr)                              */
    double alpha_pol;     /* polarisability; 0 = no polarisation potential              */
    int    pol_form;      /* 0: -a/2 (1-exp(-(r/r_c)^6))^2 / r^4 (Potentials.cpp:111-129)
                             1: -a / (2 (r^2 + r_c^2)^2)                                  */
    double r_c;           /* cutoff radius (the reference fixes 1.5 for form 0)           */
    int    n_transition;  /* > 0: explicit; 0: chi_cutoff rule (WavefunctionSetup.cpp:278-324) */
    double chi_cutoff;    /* 1e-15 in the reference                                       */
} scatt_scan_desc;

/* Policies (defaults in parentheses are the reference's). */
typedef struct {
    double W_min;                 /* (0.001) SchurInverter.hpp:74                     */
    int    stab_n_max;            /* (60)    SchurInverter.hpp:75                     */
    double shift_margin;          /* (0.01)  SchurInverter.hpp:76                     */
    int    n_asym;                /* (300)   main.cpp:1335                            */
    int    allow_closed_channels; /* (0)     AsymptoticAmplitudes.hpp:72-102          */
    int    orthogonalize;         /* (1)     DipoleMatrixElement.hpp:104-148          */
    int    max_batch;             /* energies per device batch; 0 = as many as fit    */
    int    use_graphs;            /* 1: each chunk of 8 radial steps is replayed
                                     from a CUDA graph captured once per pattern
                                     of stages (same results, fewer launches)    */
    int    diagnostics;           /* 1: S-matrix unitarity and eigenphases            */
    int    timing;                /* 1: CUDA-event timing of the solve (scatt_last_stats) */
    int    keep_window;           /* (1) keep Rinv and Sinv over the fit window and sweep psi back
                                     over it (BackPropagator.cpp:603-703), which the fit residual
                                     diagnostics need; 0: accumulate the fit forward, [A; B] =
                                     G_A(N-1)^T Z_N like the dipole rows, which drops the window
                                     store (about 1.8 GB of the 2.5 GB per energy at l_cont 20,
                                     N_t 1046) so that many more energies share each batched
                                     call; the fit residual diagnostics are then NaN */
} scatt_solve_opts;

/* Diagnostics per energy (index into scatt_outputs.diag). */
#define SCATT_DIAG_FIT_RESIDUAL_MAX    0
#define SCATT_DIAG_FIT_RESIDUAL_REL    1
#define SCATT_DIAG_A_MINUS_I_MAX       2
#define SCATT_DIAG_K_SYMMETRY_ERR_AA   3
#define SCATT_DIAG_S_UNITARITY_ERR_AA  4
#define SCATT_DIAG_K_SYMMETRY_ERR_KME  5
#define SCATT_DIAG_UNITARITY_ERR_KME   6
#define SCATT_DIAG_N_FIT_START         7
#define SCATT_DIAG_N_FIT_END           8
#define SCATT_DIAG_N_TRANSITION        9
#define SCATT_DIAG_SHIFTS_A           10
#define SCATT_DIAG_SHIFTS_S           11
#define SCATT_DIAG_N_CLOSED_L         12
#define SCATT_DIAG_SCHUR_COUPLING_0   13
#define SCATT_NDIAG                   16

/* Caller-owned host outputs; any pointer may be NULL.  Np = (l_cont_max+1)^2.
 * For energy e, a matrix output starts at e * Np * Np and is column-major
 * with ld = Np; an energy whose l_cont is smaller fills the leading block.
 * Slot order of the six dipole slices is (L,x) (L,y) (L,z) (V,x) (V,y) (V,z)
 * (DipoleWriter::slice_index). */
typedef struct {
    double* K_kme;       /* [E][Np*Np]  KMatrixExtractor::extract K                    */
    double* A;           /* [E][Np*Np]  AsymptoticAmplitudes A                         */
    double* B;           /* [E][Np*Np]  AsymptoticAmplitudes B                         */
    double* K_aa;        /* [E][Np*Np]  B A^-1                                         */
    double* b_overlap;   /* [E][Np*n_occ]  <phi_alpha | psi_beta>, Np x n_occ          */
    double* D_re;        /* [E][6][Np]  D_reduced                                      */
    double* D_im;
    double* Draw_re;     /* [E][6][Np]  D_reduced_raw                                  */
    double* Draw_im;
    double* d_raw;       /* [E][6][Np]                                                 */
    double* d_corr;      /* [E][6][n_occ]                                              */
    double* partial_sigma; /* [E][6]                                                   */
    double* eig_kme;     /* [E][Np]  eigenphases atan(eig K) (diagnostics = 1)         */
    double* eig_aa;      /* [E][Np]                                                    */
    double* diag;        /* [E][SCATT_NDIAG]                                           */
    int*    status;      /* [E]      per-energy SCATT_* status                         */
} scatt_outputs;

int scatt_ctx_create(int device, scatt_ctx** out);
int scatt_ctx_destroy(scatt_ctx* ctx);
/* Builds every energy-independent table on the device (potential Gaunt
 * pairs, exchange coupling CSR, chi, dipole rows, stability spectra). */
int scatt_upload_static(scatt_ctx* ctx, const scatt_scan_desc* desc);
/* n_transition and channel sizes of the uploaded scan: out[0] = n_transition,
 * out[1] = Np_max, out[2] = N_f, out[3] = n_lambda, out[4] = n_sigma. */
int scatt_scan_info(scatt_ctx* ctx, int* out5);
/* Solves n_energy energies E_e = energies[e] (Hartree) with continuum cutoffs
 * l_cont[e] (NULL: all l_cont_max).  Returns SCATT_OK or the first failing
 * energy's status; outputs->status has every energy's status. */
int scatt_solve_batch(scatt_ctx* ctx, int n_energy, const double* energies, const int* l_cont,
                      const scatt_solve_opts* opts, const scatt_outputs* outputs);
/* Default policies (the reference's). */
void scatt_default_opts(scatt_solve_opts* opts);

/* ------------------------------------------------------ streaming scan
 * The energy loop of the reference's driver (src/main.cpp:847-877, one
 * run_one_energy per ik) as a conveyor: energies are queued and solved in
 * `slots` device slots split into `groups` phase groups.  Every energy of a
 * group is at the same radial step; groups start staggered by 1/groups of
 * the radial sweep, so once the conveyor is full one group finishes every
 * 1/groups of a sweep and its slots take the next queued energies at once.
 * groups = 1 is the lock-step batch that scatt_solve_batch runs.
 * Each energy's results equal scatt_solve_batch's for it.  A scan holds its
 * device memory (slots sized for l_cont_max) until scatt_scan_close. */
typedef struct scatt_scan scatt_scan;
/* slots <= 0: as many as fit in 85% of free device memory;
 * 1 <= groups <= 64 (clamped to slots); l_cont_max < 0: the uploaded
 * scan's.  The scan keeps *opts as given. */
int scatt_scan_open(scatt_ctx* ctx, const scatt_solve_opts* opts, int slots, int groups,
                    int l_cont_max, scatt_scan** out);
/* Queues energies (Hartree; l_cont NULL: the scan's l_cont_max); their
 * submission indices continue from the previous submissions. */
int scatt_scan_submit(scatt_scan* scan, int n, const double* energies, const int* l_cont);
/* Runs the conveyor until at least one group finishes, then that group's
 * post stages.  The finished energies' results go to rows 0 .. *n_done - 1
 * of `outputs` (laid out as for scatt_solve_batch, capacity >= slots rows)
 * and their submission indices to index_out (may be NULL).  *n_done = 0
 * when nothing is queued or in flight.  Returns SCATT_OK or the first
 * failing energy's status (outputs->status has each one's). */
int scatt_scan_step(scatt_scan* scan, const scatt_outputs* outputs, int capacity, int* n_done,
                    long long* index_out);
/* Energies waiting in the queue and in flight in slots. */
int scatt_scan_pending(scatt_scan* scan, int* queued, int* in_flight);
/* Slot and group counts the scan was opened with. */
int scatt_scan_shape(scatt_scan* scan, int* slots, int* groups);
int scatt_scan_close(scatt_scan* scan);
/* Timing of the last scatt_solve_batch with opts.timing = 1, or of every
 * scatt_scan_step since the last scatt_scan_open (device clock, CUDA events
 * on the library stream): out[0] device seconds, out[1] seconds spent in the
 * sampled R^-1 inversions, out[2] number of sampled inversions, out[3] kernel
 * launches issued, out[4] radial-sweep seconds, out[5] post-processing
 * seconds, out[6] floating-point operations of the sampled inversions
 * (2 n^3 per matrix of order n). */
int scatt_last_stats(scatt_ctx* ctx, double* out7);

/* ------------------------------------------------------ adjoint
 * Gradients of the dipoles (and of sigma, tau built on them) with respect
 * to V(n) and the polarisation potential.  The reference has no adjoint.
 * scatt_adjoint_forward solves n_energy energies as one lock-step batch
 * (results into `outputs` as scatt_solve_batch, rows in submission order),
 * keeping Rinv(a-1) and G(a-1)^T at every segment start a (segment: a
 * positive multiple of 8 steps).  The small stages after the sweep (K
 * extraction, psi_N, the fit window, the dipole algebra) are differentiated
 * by the caller on views of the window store (scatt_adjoint_view_of; the
 * Python binding runs them in torch), which writes dJ/dRinv(n),
 * dJ/dSinv(n) (n_s <= n < N) and dJ/dG(N-1)^T into the view's cotangent
 * buffers.  scatt_adjoint_reverse then recomputes each segment from its
 * checkpoint and walks it backward: vtr (host, n_energy x Nr, may be NULL)
 * receives tr dJ/dV(n) per energy, vfull (device [Nr][Np_max][Np_max],
 * may be NULL) accumulates dJ/dV(n) summed over the energies.  The terms
 * of V(N) itself (the outer boundary) stay with the caller's small stages.
 * One reverse pass per forward.  Matrices are column-major. */
typedef struct scatt_adjoint scatt_adjoint;
typedef struct {
    int N, n_s, n_window, n_tr, n_pts, n_start, ne_fit;
    int Np, Nt, Nf, Krows, Np_max, l_cont;
    double E;
    double* Rwin;          /* (N - n_s + 1) x Nt x Nt: Rinv(n_s + i) */
    double* Swin;          /* (N - n_s + 1) x Np x Np: Sinv(n_s + i) */
    double* G_last;        /* Krows x Nt: G(N-1)^T */
    double* RBwin;         /* n_window x Nt x Nt: dJ/dRinv(n_s + i), zero after the forward */
    double* SBwin;         /* n_window x Np x Np: dJ/dSinv(n_s + i) */
    double* GB_last;       /* Krows x Nt: dJ/dG(N-1)^T */
    const double* V_N;     /* Np_max x Np_max: V(N) */
    const double* B_N;     /* Np_max x Nf */
    const double* Bs_N;    /* Np_max x Nf: B(N) D^-1(N) */
    const double* C_N;     /* Krows x Np_max dipole rows at N, NULL when N is past them */
    const double* Bs_win;  /* n_window x Np_max x Nf: Bs(n_s + i) (zero outside the exchange
                              region), NULL when no window step is inside it */
} scatt_adjoint_view;

/* Polarisation potential V_pol(alpha, r_c) of the uploaded scan (form as in
 * scatt_scan_desc) and an optional additive perturbation of V: a DEVICE
 * array [Nr][Np_max][Np_max] (column-major per n, upper triangle read,
 * NULL: none) that stays the caller's and must outlive its use. */
int scatt_set_polarization(scatt_ctx* ctx, double alpha, double r_c, int pol_form);
int scatt_set_potential_delta(scatt_ctx* ctx, const double* dV_device);
int scatt_adjoint_forward(scatt_ctx* ctx, const scatt_solve_opts* opts, int n_energy, const double* energies,
                          const int* l_cont, int segment, const scatt_outputs* outputs, scatt_adjoint** out);
int scatt_adjoint_view_of(scatt_adjoint* adj, int i, scatt_adjoint_view* view);
int scatt_adjoint_reverse(scatt_adjoint* adj, double* vtr, double* vfull_device);
int scatt_adjoint_close(scatt_adjoint* adj);

/* ------------------------------------------------------ psi reconstruction
 * BackPropagator::run + get_psi (src/scatt/BackPropagator.cpp:199-802):
 * psi(n) = (W^-1(n) Z_n)_psi with Z_n = Rinv(n) Z_{n+1} from the outer
 * boundary Z_N, over any range n_lo <= n < n_hi of the grid (the reference
 * keeps [0, n_transition) and the 300-point asymptotic tail).  Solves
 * n_energy energies as one lock-step batch (results into `outputs` as
 * scatt_solve_batch, with the fit accumulated forward: keep_window and
 * use_graphs of `opts` are ignored), keeping Rinv(a - 1) at every segment
 * start a, then sweeps back from N - 1 to n_lo, recomputing each segment's
 * Sinv and Rinv from its checkpoint.  psi(n) of energy i (submission order)
 * lands at psi_out + (i * (n_hi - n_lo) + n - n_lo) * Np_max^2, column-major
 * Np x Np with ld Np_max (zero outside an energy's own Np x Np block).
 * psi_out is host memory; when it is page-locked the copies of one segment
 * run while the next segment is recomputed.  segment: a positive multiple of
 * 8 radial steps.  Device memory per energy, besides the scan state: about
 * (Nr / segment + segment) N_t^2 + segment (Np^2 + 2 Np_max^2) doubles. */
int scatt_psi_sweep(scatt_ctx* ctx, const scatt_solve_opts* opts, int n_energy, const double* energies,
                    const int* l_cont, int segment, int n_lo, int n_hi, const scatt_outputs* outputs,
                    double* psi_out);

/* The on-disk psi store of the reference's back-propagation, the files its
 * continuum-continuum dipole driver reads (src/scatt/BackPropagator.cpp:
 * 27-101, :255-283, :700-745; the full-matrix PotentialStorage layout of
 * src/scatt/PotentialStorage.cpp:31-35, :556-631, :1542-1566): a directory
 * of pot_chunk_<c>.bin (int32 count + count column-major N_psi x N_psi
 * matrices), metadata.bin (size_t points, int32 N_psi, chunk_size,
 * chunks), psi_asym.bin (the asymptotic buffer, 32-byte 'PSI_ASYM'
 * header), manifest.txt (the reference's "kind=psi energy=... keep=lo..hi"
 * line) and __SUCCESS__ written last.  Host-only.
 * scatt_psi_store_write: psi holds the keep_hi - keep_lo + 1 matrices of
 * points keep_lo .. keep_hi, ld^2 apart with leading dimension ld (as
 * scatt_psi_sweep writes them, ld = Np_max); psi_asym likewise the n_asym
 * matrices of points asym_offset .. asym_offset + n_asym - 1 (NULL when
 * n_asym = 0).  scatt_psi_store_dirname: the reference's default directory
 * name.  The reader refuses a store without __SUCCESS__;
 * scatt_psi_store_info: out6 = points, N_psi, chunk_size, chunks, n_asym,
 * asym_offset; scatt_psi_store_read: matrices first .. first + count - 1
 * (counted from keep_lo), packed N_psi x N_psi. */
typedef struct {
    double energy, dr;
    int n_grid, n_psi, n_f, l_cont, l_exch, n_occ, n_transition;
    int keep_lo, keep_hi, chunk_size, n_asym, asym_offset;
} scatt_psi_store_meta;
typedef struct scatt_psi_store scatt_psi_store;
int scatt_psi_store_dirname(const scatt_psi_store_meta* meta, char* buf, int cap);
int scatt_psi_store_write(const char* dir, const scatt_psi_store_meta* meta, const double* psi, int ld,
                          const double* psi_asym, int ld_asym);
int scatt_psi_store_open(const char* dir, scatt_psi_store** out);
int scatt_psi_store_info(scatt_psi_store* h, long long* out6);
int scatt_psi_store_manifest(scatt_psi_store* h, char* buf, int cap);
int scatt_psi_store_read(scatt_psi_store* h, long long first, long long count, double* out);
int scatt_psi_store_read_asym(scatt_psi_store* h, double* out);
int scatt_psi_store_close(scatt_psi_store* h);

/* Continuum-continuum dipole, the consumer of the psi store
 * (postprocessing/two_photon_delay/cc_dipole/src/CCDipole.cpp:294-334 and
 * its range-accumulating API, include/CCDipole.hpp): for one final state
 * kappa and n_nu intermediate states nu, length gauge,
 *   cc_nu[beta, alpha] = sum_i w_i r_i psi_kappa(i)[:, beta]^T A^q psi_nu(i)[:, alpha]
 * over the radial points ir0 .. ir0 + n_pts - 1 (n_pts >= 5), r_i =
 * (ir0 + i + 1) dr (r_min = dr, CCDipole.cpp:236), w_i the window's Simpson
 * weights (:100-122), A^q = sqrt(4 pi / 3) gaunt_real(l_mu, m_mu, 1, q,
 * l_nu, m_nu) with q = +1 / -1 / 0 for x / y / z (:135-160).  psi_kappa:
 * n_pts column-major n_mu x n_mu matrices with leading dimension ld, ld^2
 * apart (one energy of scatt_psi_sweep's output, ld = Np_max); psi_nu: n_nu
 * such stacks one after another; cc: n_nu column-major n_mu x n_mu
 * matrices (ld n_mu).  Host buffers; the points stream through the device
 * in chunks, each psi_kappa chunk read once for all nu. */
int scatt_cc_dipole(int n_mu, int ld, int n_pts, int ir0, double dr, int q, const double* psi_kappa,
                    int n_nu, const double* psi_nu, double* cc);

/* ------------------------------------------------------ preprocessing
 * Hartree potential from the density's single-centre multipoles by the
 * radial Poisson integrals (preprocessing/src/potential/Hartree.hpp:71-246,
 * build_V_H):  V_lm(r) = 4 pi / (2l + 1) [ r^-(l+1) int_0^r rho_lm r'^(l+2)
 * + r^l int_r^R rho_lm r'^(1-l) ] on r_k = r0 + k dr, k < Nr, with the
 * cumulative integrator of preprocessing/src/sce/RadialGrid.hpp:84-100 and
 * the reference's guards (channels above the overflow-safe l or with
 * max |rho_lm| < 1e-12 stay 0; non-finite values become 0; V_00(0) =
 * 4 pi int rho_00 r').  rho_lm: n_rows >= (l_max + 1)^2 rows of Nr points,
 * row-major (channel idx = l^2 + l + m); V_H: (l_max + 1)^2 rows of Nr,
 * row-major -- the layout scatt_scan_desc.V_H takes.  Host buffers. */
int scatt_hartree(int l_max, int n_rows, int Nr, double r0, double dr, const double* rho_lm, double* V_H);

/* Single-centre expansion (preprocessing/src/sce/SCE.hpp:122-266, project):
 * F_lm(r_k) = int F(r_k, Omega) Y^R_lm(Omega) dOmega, l <= Lmax, on the grid
 * of preprocessing/src/angular/Grid.hpp: n_theta = Lmax + 1 Gauss-Legendre
 * nodes in cos(theta), ascending; n_phi = 2 (Lmax + 1) nodes
 * phi_j = 2 pi j / n_phi.  scatt_sce_grid returns the grid (cos_theta and
 * weights: n_theta each; phi: n_phi), host-only.  scatt_sce_project takes
 * the samples F(r_k, theta_i, phi_j) at samples[(k n_theta + i) n_phi + j]
 * for Nr radial points and writes F_lm row-major [(Lmax + 1)^2][Nr]
 * (channel l^2 + l + m, Y^R of SCE.hpp:11-15).  The Fourier and Legendre
 * steps run as DMMA GEMMs over chunks of `chunk` radial points (<= 0:
 * chosen to hold a chunk's buffers in 512 MB).  Host buffers. */
int scatt_sce_grid(int Lmax, double* cos_theta, double* weights, double* phi);
int scatt_sce_project(int Lmax, int Nr, int chunk, const double* samples, double* F_lm);
/* The molecular orbitals and the density of a contracted spherical-Gaussian
 * basis, sampled on the same grid around `origin` (radial points
 * r_k = r0 + k dr, k < Nr) and projected: the reference's build_basis /
 * evaluate_mo / evaluate_density (preprocessing/src/basis/MoldenBasis.hpp:
 * 48-229, the normalisation of SphericalGaussian.hpp and Primitive.hpp)
 * followed by project.  Shell i: centre shell_center[3i..3i+2] (bohr),
 * angular momentum shell_l[i], shell_nprim[i] primitives whose exponents
 * and raw contraction coefficients follow the previous shells' in exps /
 * coefs; its 2l + 1 AOs in molden order (p: m = +1, -1, 0; l >= 2:
 * m = 0, +1, -1, +2, -2, ...).  C: n_mo x nbf row-major MO coefficients,
 * occ: n_mo occupations.  vx_form: 0 none, 1 the Slater local exchange
 * -(3/pi)^(1/3) rho^(1/3), 2 the Kohn-Sham one, 1.5 times that
 * (preprocessing/src/potential/LocalExchange.hpp), projected into vx_lm
 * (given exactly when vx_form != 0).  orb_lm: [n_mo][(Lmax + 1)^2][Nr],
 * rho_lm and vx_lm: [(Lmax + 1)^2][Nr] (orb_lm and rho_lm may be NULL).
 * The AO values (a kernel per point and shell), the orbitals (Phi^T C^T, a
 * DMMA GEMM), the density, the local exchange and the projections run on
 * the device over chunks of `chunk` radial points (<= 0: automatic).
 * Host buffers. */
int scatt_sce_basis(int Lmax, int Nr, double r0, double dr, const double* origin, int n_shell, const int* shell_l,
                    const int* shell_nprim, const double* shell_center, const double* exps, const double* coefs,
                    int n_mo, const double* C, const double* occ, int vx_form, int chunk, double* orb_lm,
                    double* rho_lm, double* vx_lm);

/* Molden reader (preprocessing/src/molden/Molden.hpp), host-only: the
 * [Atoms] (bohr; Angs or unmarked blocks converted), [GTO] and [MO]
 * sections and the [5D] / [5D7F] / [5D10F] / [7F] / [9G] flags, kept as
 * written.  scatt_molden_info: out7 = n_atoms, n_shell, nbf, alpha MOs,
 * beta MOs, primitives in all, Cartesian shells of l >= 2.
 * scatt_molden_atoms: n_atoms x (Z, x, y, z).  scatt_molden_shells: the
 * arrays scatt_sce_basis takes (l, primitives, centre, exponents and raw
 * coefficients in file order); a Cartesian shell of l >= 2 is an error, as
 * in the reference's build_basis.  scatt_molden_mos: n_mo x nbf
 * coefficients (row-major, AO order), occupations and energies of the alpha
 * (beta = 0) or beta orbitals.  Malformed files return SCATT_ERR_IO with
 * the offending line. */
typedef struct scatt_molden scatt_molden;
int scatt_molden_open(const char* path, scatt_molden** out);
int scatt_molden_info(scatt_molden* m, int* out7);
int scatt_molden_atoms(scatt_molden* m, double* zxyz);
int scatt_molden_shells(scatt_molden* m, int* l, int* nprim, double* center, double* exps, double* coefs);
int scatt_molden_mos(scatt_molden* m, int beta, double* C, double* occ, double* energy);
int scatt_molden_close(scatt_molden* m);

/* ------------------------------------------------------ file formats
 * Host-only entry points (no device work, no GPU needed) for the files
 * around the path, on an HDF5 subset written from the public file-format
 * specification (the container has no libhdf5): superblock 0, symbol-table
 * groups, version-1 object headers, contiguous or chunked + deflate
 * datasets, scalar attributes.  Readers also take superblock 1, continuation
 * blocks, compact layout, shuffle and fletcher32; anything else returns
 * SCATT_ERR_IO with the reason, never a misread. */

/* Generic writer: the file appears at `path` on scatt_h5w_close(h, 1)
 * (written as path.tmp.pid<PID>, then renamed); keep = 0 discards it.
 * kind: 0 f64, 1 i64, 2 i32; rank 0 = scalar; data row-major; gzip 1..9
 * stores the dataset chunked along its first dimension and deflated. */
typedef struct scatt_h5w scatt_h5w;
int scatt_h5w_open(const char* path, scatt_h5w** out);
int scatt_h5w_group(scatt_h5w* h, const char* path);
int scatt_h5w_dataset(scatt_h5w* h, const char* path, int kind, int rank, const long long* dims,
                      const void* data, int gzip);
int scatt_h5w_attr_f64(scatt_h5w* h, const char* obj, const char* name, double v);
int scatt_h5w_attr_i64(scatt_h5w* h, const char* obj, const char* name, long long v);
int scatt_h5w_attr_str(scatt_h5w* h, const char* obj, const char* name, const char* v);
int scatt_h5w_close(scatt_h5w* h, int keep);

/* Generic reader.  kind: 0 absent, 1 group, 2 dataset.  shape: rank,
 * dims (<= 8) and element kind (0 float, 1 integer, 3 string).  read: the
 * block [start, start + count) (both NULL: everything) converted to f64
 * (as_int = 0) or int64, row-major.  list: member names, one per line.
 * attr: kind 0 absent, 1 float, 2 integer-valued, 3 string. */
typedef struct scatt_h5r scatt_h5r;
int scatt_h5r_open(const char* path, scatt_h5r** out);
int scatt_h5r_kind(scatt_h5r* h, const char* path, int* kind);
int scatt_h5r_shape(scatt_h5r* h, const char* path, int* rank, long long* dims8, int* elem_kind);
int scatt_h5r_read(scatt_h5r* h, const char* path, int as_int, int rank, const long long* start,
                   const long long* count, void* out);
int scatt_h5r_list(scatt_h5r* h, const char* group, char* buf, long long cap, long long* needed);
int scatt_h5r_attr(scatt_h5r* h, const char* obj, const char* name, int* kind, double* f, long long* i,
                   char* s, long long cap);
int scatt_h5r_close(scatt_h5r* h);

/* Dipole scan output in the layout of the reference's DipoleWriter
 * (src/scatt/DipoleIO.hpp:115-148, DipoleIO.cpp:141-336): <scan_dir>/
 * manifest.h5 (/grid, /kgrid attributes; /occ, /atoms datasets;
 * /conventions, /run string attributes), one ik<NNNN>.h5 per energy (/meta
 * attributes ik, k = ik dk, E = k^2 / 2, omega = E - E_HOMO,
 * fit_residual_rel, K_symmetry_err; /A, /B (n_ch x n_ch), /b_overlap
 * (n_ch x n_occ), /dipole/{length,velocity}/{x,y,z}/{D_ortho_re,
 * D_ortho_im, D_raw_re, D_raw_im, d_raw, d_correction} + attribute
 * partial_sigma) and __SUCCESS__ from finalize.  Files are written under a
 * PID-tagged temporary name and renamed into place; a rename that loses to
 * another process's identical file counts as success. */
typedef struct {
    double r_min, dr;
    long long N_grid;
    int    l_max_continuum;
    double dk;
    int    ik_min, ik_max;           /* ik_max exclusive */
    double E_HOMO;                   /* initial-state energy (Koopmans) */
    int    n_occ;
    const double* occ_energies;      /* n_occ */
    const double* occ_spin_factors;  /* n_occ */
    int    n_atoms;
    const int* Z;                    /* n_atoms */
    const double* xyz_bohr;          /* n_atoms x 3 */
    const char* molecule_name;       /* NULL: "" */
    const char* git_hash;
    const char* iso_date_utc;
    const char* psi_dir_prefix;
} scatt_dipole_meta;

/* One energy's payload; matrices row-major in their natural orientation,
 * slices in the order length x, y, z, velocity x, y, z. */
typedef struct {
    int ik, n_ch, n_occ;
    const double *A, *B;             /* n_ch x n_ch */
    const double* b_overlap;         /* n_ch x n_occ */
    const double *D_re, *D_im;       /* 6 x n_ch, orthogonalised */
    const double *Draw_re, *Draw_im; /* 6 x n_ch */
    const double* d_raw;             /* 6 x n_ch */
    const double* d_corr;            /* 6 x n_occ */
    const double* partial_sigma;     /* 6 */
    double fit_residual_rel, K_symmetry_err;
} scatt_dipole_energy;

/* Creates scan_dir and its manifest (kept as it is when present: a resumed scan). */
int scatt_dipole_open(const char* scan_dir, const scatt_dipole_meta* meta);
int scatt_dipole_has_energy(const char* scan_dir, int ik, int* has);
int scatt_dipole_write_energy(const char* scan_dir, const scatt_dipole_meta* meta, const scatt_dipole_energy* e);
int scatt_dipole_finalize(const char* scan_dir);

/* Preprocessing input in the reference's schema (src/io/HDF5Reader.hpp:
 * 42-86, 446-570): a path ending in .orbitals.h5 or .potentials.h5 whose
 * sibling exists opens the split layout (orbitals + initial state from one
 * file, potential + polarizability from the other), anything else one
 * combined file.  info: out_i = {Nr, Lmax_sce, n_alpha, n_occ_alpha, n_sce,
 * Nlm_orb_store, Nr_orb_store, has_initial_state}, out_d = {rmin, dr,
 * initial-state energy, alpha_iso (0 when absent)}.  desc fills a scan
 * description for continuum cutoff l_cont_max with the rows the reference
 * reads (V_H: (2 l + 1)^2 multipoles; orbitals: (l + min(l, 10) + 1)^2
 * channels, main.cpp:365, 700-721), pointing into memory the handle owns
 * until close or the next desc; an /initial_state SOMO becomes orbital
 * n_sce and the dipole initial state (main.cpp:787-808), else the HOMO.
 * *E_init (may be NULL) receives that state's energy. */
typedef struct scatt_preproc scatt_preproc;
int scatt_preproc_open(const char* path, scatt_preproc** out);
int scatt_preproc_info(scatt_preproc* p, int* out_i8, double* out_d4);
int scatt_preproc_orbital_energies(scatt_preproc* p, double* out, int n);
int scatt_preproc_atoms(scatt_preproc* p, double* out4, int n);
int scatt_preproc_desc(scatt_preproc* p, int l_cont_max, scatt_scan_desc* desc, double* E_init);
int scatt_preproc_close(scatt_preproc* p);

#ifdef __cplusplus
}
#endif

#endif /* SCATT_B200_H */
