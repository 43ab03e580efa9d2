/*
 * quick_b200 C ABI.
 *
 * Part 1 is a drop-in for the Fortran-callable bridge of QUICK's CUDA build
 * (src/cuda/gpu.h:16-58, implemented in src/cuda/gpu.cu).  Same symbol names
 * (lower case + trailing underscore), every argument by pointer (Fortran
 * by-reference), arrays column-major, indices stored inside arrays 1-based,
 * void return.  The call order QUICK's Fortran uses is kept:
 *   start-up   gpu_startup_ -> gpu_set_device_ -> gpu_init_ -> gpu_setup_
 *              -> gpu_upload_xyz_ -> gpu_upload_atom_and_chg_
 *              -> gpu_upload_basis_ -> gpu_upload_cutoff_matrix_
 *   per SCF    gpu_upload_method_ -> gpu_upload_calculated_
 *              -> gpu_upload_cutoff_ -> gpu_get2e_        (src/hfoperator.f90:76-98)
 *   gradient   gpu_upload_calculated_ -> gpu_upload_cutoff_ -> gpu_upload_grad_
 *              -> gpu_grad_                               (src/gradient.f90:279-286)
 *   DFT        ... -> gpu_getxc_                          (src/dft.f90:893-899)
 * Where QUICK prints and exits on a fault, these print to stderr and record
 * a sticky error that qb_status() returns.
 *
 * Part 2 adds entry points QUICK does not have (int status return, 0 = ok).
 */
#ifndef QUICK_B200_H
#define QUICK_B200_H
#ifdef __cplusplus
extern "C" {
#endif

/* ---- Part 1: QUICK's gpu_* bridge ------------------------------------ */
/* src/cuda/gpu.cu:29 */
void gpu_startup_(void);
/* src/cuda/gpu.cu:18 */
void gpu_set_device_(int* gpu_dev_id);
/* src/cuda/gpu.cu:43-173 */
void gpu_init_(void);
/* src/cuda/gpu.cu:206-215 */
void gpu_shutdown_(void);
/* src/cuda/gpu.cu:175-201 (device count, id, memory MB, SM count, clock GHz, name, name length, major, minor) */
void gpu_get_device_info_(int* gpu_dev_count, int* gpu_dev_id, int* gpu_dev_mem, int* gpu_num_proc,
                          double* gpu_core_freq, char* gpu_dev_name, int* name_len, int* majorv, int* minorv);
/* src/cuda/gpu.cu:221-267 */
void gpu_setup_(int* natom, int* nbasis, int* nElec, int* imult, int* molchg, int* iAtomType);
/* src/cuda/gpu.cu:269-278: 0 HF, 1 B3LYP (exchange 0.2), 2 DFT (no exchange) */
void gpu_upload_method_(int* quick_method);
/* src/cuda/gpu.cu:283-328: xyz(3, natom) in bohr */
void gpu_upload_xyz_(double* atom_xyz);
/* src/cuda/gpu.cu:334-349 */
void gpu_upload_atom_and_chg_(int* atom, double* atom_chg);
/* src/cuda/gpu.cu:1070-1390 */
void gpu_upload_basis_(int* nshell, int* nprim, int* jshell, int* jbasis, int* maxcontract,
                       int* ncontract, int* itype, double* aexp, double* dcoeff,
                       int* first_basis_function, int* last_basis_function,
                       int* first_shell_basis_function, int* last_shell_basis_function,
                       int* ncenter, int* kstart, int* katom, int* ktype, int* kprim, int* kshell,
                       int* Ksumtype, int* Qnumber, int* Qstart, int* Qfinal, int* Qsbasis, int* Qfbasis,
                       double* gccoeff, double* cons, double* gcexpo, int* KLMN);
/* src/cuda/gpu.cu:401-1003: YCutoff(nshell, nshell), cutPrim(jbasis, jbasis); builds the
   shell-pair list in QUICK's exact order */
void gpu_upload_cutoff_matrix_(double* YCutoff, double* cutPrim);
/* src/cuda/gpu.cu:1008-1065: O(nbasis, nbasis) holds the one-electron operator, dense the density */
void gpu_upload_calculated_(double* o, double* co, double* vec, double* dense);
/* src/cuda/gpu.cu:356-394.  Fortran callers pass three arguments
   (src/hfoperator.f90:81); the fourth is never read, DMCutoff is 1e-9 as in QUICK. */
void gpu_upload_cutoff_(double* cutMatrix, double* integralCutoff, double* primLimit, double* DMCutoff);
/* src/cuda/gpu.cu:1806-1864: o <- o + J - (h/2) K, symmetric */
void gpu_get2e_(double* o);
/* src/cuda/gpu.cu:1393-1444: grad(3 natom) accumulates, gradCutoff */
void gpu_upload_grad_(double* grad, double* gradCutoff);

/* Declared in QUICK's src/cuda/gpu.h:31 and defined nowhere in QUICK (no caller): kept for a
   complete drop-in; stores the energy, which nothing here reads. */
void gpu_upload_energy_(double* E);
/* src/cuda/gpu.cu:1481-1551: grad <- grad + two-electron gradient */
void gpu_grad_(double* grad);
/* src/cuda/gpu.cu:1866-1975: XC quadrature on QUICK's SG1 grid for the method of the last
   gpu_upload_method_ (1 = B3LYP, 2 = BLYP).  Eelxc, aelec and belec are accumulated into; o is
   overwritten with the symmetrised lower triangle of (O as uploaded by gpu_upload_calculated_ +
   V_xc).  isg = 1 is QUICK's SG1 grid; isg = 2 (no counterpart in QUICK's GPU path) is a
   75-radial (Euler-Maclaurin) x 302-point (Lebedev-Laikov) grid per atom with Becke's fuzzy-cell
   partition.  isg = 0 is rejected: QUICK's GPU path generates no SG0 points. */
void gpu_getxc_(int* isg, double* sigrad2, double* Eelxc, double* aelec, double* belec, double* o);
/* src/cuda/gpu.cu:1446-1479 */
void gpu_cleanup_(void);
/* src/cuda/gpu.cu:1991-2237: QUICK's conventional (stored-integral) SCF.  Computes every unique
   integral (ij|kl) of the shell quartets with Y_ij Y_kl > leastIntegralCutoff and writes those
   with |(ij|kl)| > maxIntegralCutoff to intFileName (blank-terminated, as Fortran passes it) in
   QUICK's format: blocks of 150000 records written as int IJ[], int KL[], double value[] (the
   last block short), IJ = i nbasis + j, KL = k nbasis + l, 0-based, i <= j, k <= l,
   (i, j) <= (k, l), cons-scaled values.  intNum += the number written.  s, p, d and f shells.
   Replaces the density screen, so gpu_upload_cutoff_ must precede the next two-electron
   build. */
void gpu_aoint_(double* leastIntegralCutoff, double* maxIntegralCutoff, int* intNum, char* intFileName);
/* src/cuda/gpu.cu:1559-1801: o <- symmetric (O as uploaded + J - (h/2) K) from the intindex
   stored integrals of intFileName and the density of the last gpu_upload_calculated_ (h from
   gpu_upload_method_), as gpu_get2e_ returns it. */
void gpu_addint_(double* o, int* intindex, char* intFileName);

/* ---- Part 2: additions ---------------------------------------------- */
/* Sticky status of the bridge: 0 ok, else an error code; message via qb_last_error. */
int qb_status(void);
const char* qb_last_error(void);
void qb_clear_error(void);

/* Run subsequent work on this CUDA stream (a cudaStream_t), 0 = the bridge's own stream. */
int qb_set_stream(void* stream);

/* QUICK's shell-pair list as gpu_upload_cutoff_matrix_ built it: xy[2*i], xy[2*i+1] are the
   sorted-Qshell indices of pair i (QUICK's sorted_YCutoffIJ, gpu.cu:447-647); also the sorted
   shell order (sorted_Q, sorted_Qnumber, gpu.cu:1191-1218) and fStart / ffStart.
   Returns the number of pairs (or -1 if cap is too small). */
int qb_get_pairlist(int* xy, int cap, int* sorted_Q, int* sorted_Qnumber, int qcap, int* fStart, int* ffStart);

/* Host-only: QUICK's pair-list construction on given inputs, without a GPU (for tests).
   sorted_Q, sorted_Qnumber, kprim are 0-based Qshell data; YCutoff is (nshell, nshell). */
int qb_build_pairlist_host(int Qshell, const int* sorted_Q, const int* sorted_Qnumber, const int* kprim,
                           int nshell, const double* YCutoff, int* xy_out, int cap, int* fStart, int* ffStart);

/* Schwarz bounds on the GPU from the uploaded basis and coordinates, in QUICK's definition
   (src/schwarz.f90:12-548): YCutoff(nshell, nshell), cutPrim(jbasis, jbasis). */
int gpu_schwarz_(double* YCutoff, double* cutPrim);

/* Fock build on device-resident data: D (nbasis^2, device pointer), O_in and O_out (device
   pointers, may alias).  Uses the cutoffs and density screen from the last gpu_upload_cutoff_.
   Asynchronous: the work is enqueued on the library stream (qb_set_stream) and O_out is valid
   once that stream has been synchronised.  After one call with the same molecule and cutoffs
   (which sizes the quartet lists and builds the per-class tables) the call allocates nothing and
   waits for nothing, so it can be captured into a CUDA graph and replayed; the density and
   cutMatrix buffers it reads are the ones given / last uploaded. */
int qb_fock_device(const double* d_dense, const double* d_o_in, double* d_o_out);

/* No counterpart in QUICK.  The same Fock build as qb_fock_device for callers that cannot
   allocate GPU memory while they run (a host program whose pool allocator owns the device
   memory, or code that must not allocate after its set-up): it calls no cudaMalloc/cudaFree
   and takes its working memory from one fixed 64 MiB array compiled into the library, present
   on every GPU that loads it until the process exits.  Molecules whose density, Fock
   accumulator and screened quartet lists do not fit are rejected with an error (use
   qb_fock_device).  The device programs of the f-shell classes that run the generic kernel
   are copied into the same array.  The first call on a device looks up the array's device
   address (with the session's device current).  Every call waits for the library stream twice
   and copies the class counts to host memory, so no call can be recorded into a CUDA graph.
   Every quartet runs in FP64: the mixed split of qb_set_mixed_precision is not applied here.
   Calls share the array: calls that overlap on the GPU race and must not be made.  Tables
   uploaded earlier (gpu_upload_basis_, gpu_upload_cutoff_matrix_, gpu_upload_cutoff_) are used
   as they are. */
int qb_fock_device_static(const double* d_dense, const double* d_o_in, double* d_o_out);

/* Statistics of the last Fock build: unique shell quartets evaluated (one per unordered pair of
   kept shell pairs that passes QUICK's Schwarz and density tests), device time of the class
   kernels in ms, device time of the screening in ms. */
int qb_last_fock_stats(long long* quartets, double* ms_eri, double* ms_screen);

/* Statistics of the last gpu_grad_: shell quartets differentiated and the device time of the
   gradient class kernels in ms. */
int qb_last_grad_stats(long long* quartets, double* ms);

/* Mixed precision for the following Fock builds and gradients (no counterpart in QUICK, which
   is FP64 throughout): shell quartets whose bound Y_ab Y_cd DNMax (QUICK's own screening
   product, gpu_get2e_subs.h:323-328) is below cut run their Boys function, recurrences,
   contraction and density products in FP32; the others, and all accumulation into the Fock
   matrix or the gradient, stay FP64.  Classes with an f shell and L sum >= 7 run their FP32
   list in FP64.  cut = 0 (the default) keeps every quartet in FP64. */
int qb_set_mixed_precision(double cut);

/* The last Fock build's shell quartets by precision. */
int qb_last_fock_split(long long* quartets_fp64, long long* quartets_fp32);

/* XC quadrature on device pointers (no counterpart in QUICK; gpu_getxc_ without the host
   round trip): adds V_xc to the lower triangle of d_vxc (column-major nbasis^2, V(j, i) for
   j >= i; not zeroed here) for the density d_dense, and returns the grid sums of the energy
   density and of the alpha density.  sigrad2 is a host array (nbasis), as for gpu_getxc_. */
int qb_xc_device(const double* d_dense, const double* sigrad2, double* d_vxc, double* exc, double* nalpha);

/* Reproducible Fock builds (no counterpart as a switch in QUICK, whose GPU build always
   accumulates this way, gpu_common.h:115): on = 1 rounds every Coulomb and exchange
   contribution to a 64-bit fixed-point number of 1e-16 units and adds it with integer atomics,
   so the Fock matrix is bit-identical whatever the order the quartets run in (lane groups,
   streams, the screen's list order); on = 0 (default) adds doubles.  Applies to gpu_get2e_,
   qb_fock_device, qb_fock_device_static and the batched build; gradients stay FP64. */
int qb_set_fixed_point(int on);

/* Grid of the following qb_xc_device / qb_xc_grad_device calls: 1 = SG1 (default), 2 = the
   75 x 302 Becke grid (gpu_getxc_'s isg = 2).  No counterpart in QUICK. */
int qb_set_xc_grid(int grid);

/* The exchange-correlation term of the nuclear gradient (no counterpart in QUICK: its DFT
   gradient is commented out, src/optimize.f90:175): adds dE_xc/dR (3 natom, Eh/bohr) to d_grad
   for the density d_dense (device, column-major nbasis^2, total density), the functional of the
   last gpu_upload_method_ and the grid of qb_set_xc_grid.  The grid moves with the atoms: the
   basis-centre terms, the terms of the points moving with their atom and the derivatives of the
   partition weights (SSW or Becke) are all included, so the result is the derivative of the
   energy qb_xc_device integrates.  Synchronises the library stream. */
int qb_xc_grad_device(const double* d_dense, const double* sigrad2, double* d_grad);

/* Statistics of the last XC quadrature: grid points kept (weight above 1e-9), point chunks
   with at least one significant basis function, device time of the per-call phase in ms, and
   of the grid build in ms (0 when the grid was reused). */
int qb_last_xc_stats(long long* npts, long long* nchunks, double* ms, double* ms_grid);

/* Algorithmic work of the last XC quadrature, summed over its point chunks (P points, nb
   significant functions each): bytes = P nb x 32 (phi and grad phi) + 2 nb^2 x 8 (density and
   operator tiles), flops = 4 P nb^2 (density and operator contractions), gemm_flops = the
   6 P nb^2 the two triangular products and the operator DGEMM execute. */
int qb_last_xc_work(double* bytes, double* flops, double* gemm_flops);

/* The kept grid points (x, y, z, weight per point) of the last XC grid build; copies up to cap
   points and returns the number of points. */
long long qb_xc_grid(double* xyzw, long long cap);

/* The closed-shell functional (method 1 = B3LYP, 2 = BLYP) evaluated on the GPU at n pairs
   (rho = total density, sigma = |grad rho|^2), host arrays: out[3k] = f,
   out[3k+1] = df/drho, out[3k+2] = 4 df/dsigma (QUICK's b3lyp_e / b3lypf and becke/lyp). */
int qb_xc_functional(int method, int n, const double* rho, const double* sigma, double* out);

/* No counterpart in QUICK.  Autotunes the lanes per shell quartet of each straight-line Fock
   class: after a Fock build (gpu_get2e_ or qb_fock_device) or a gradient, times every compiled
   variant of every class on that call's quartet lists (into a scratch matrix; the Fock matrix
   is untouched) and keeps the fastest for the following builds.  A variant is a lane-group
   size (1, 2, 4, ... lanes per quartet), or 256 + lanes for the FP64 kernels of the classes
   with total angular momentum <= 2 that first stage the Boys-function records in shared
   memory.  After an all-FP64 call
   it tunes the FP64 class kernels, after a call with the mixed split (qb_set_mixed_precision)
   the FP32 ones on the FP32 lists.  The choice stays for the rest of the session, later
   molecules included (gpu_shutdown_ forgets it).  Writes the chosen variants, one per class, to
   groups (cap entries at most).  Synchronises the library stream. */
int qb_autotune_classes(int* groups, int cap);

/* No counterpart in QUICK.  Sets the variant of every straight-line class (n = the number of
   classes, one code each, as qb_autotune_classes writes them) for the FP64 kernels (fp32 = 0)
   or the FP32 kernels of the mixed split (fp32 = 1), as if tuned: a saved choice reused, or a
   test that runs one variant.  After gpu_upload_basis_; a code that is not a variant of its
   class is an error (status 1) and changes nothing. */
int qb_set_class_groups(const int* groups, int n, int fp32);

/* No counterpart in QUICK.  The gradient counterpart of qb_autotune_classes: after a gradient
   call (gpu_grad_ or qb_grad_device), times every compiled lanes-per-quartet size (1, 2, 4) of
   the gradient kernels of the classes with total angular momentum <= 2 on that call's quartet
   lists (into a scratch gradient) and keeps the fastest for the session's later gradients; the
   FP32 kernels after a call with the mixed split.  Writes the chosen sizes, one per class, to
   groups (cap entries at most).  Synchronises the library stream. */
int qb_autotune_grad(int* groups, int cap);

/* No counterpart in QUICK.  Passes per Fock build or gradient: the screened quartet lists are
   written in passes over disjoint ranges of bra pairs when the whole list (16 bytes a quartet)
   would take more than the list budget, QB_LIST_BUDGET_MB megabytes or else 35% of the free
   device memory when the lists are sized (at the first build after a change of cutoff or
   molecule).  Returns the current count (1: one pass).  The stored-integral path (gpu_aoint_)
   needs one pass and reports an error otherwise. */
int qb_list_passes(void);

/* No counterpart in QUICK.  Sets the lanes per quartet of every gradient class (n = the number
   of classes; 1, or 2 and 4 where qb_autotune_grad may choose them) for the FP64 or the FP32
   kernels, as if tuned.  A size that is not compiled for its class is an error (status 1) and
   changes nothing. */
int qb_set_grad_groups(const int* groups, int n, int fp32);

/* No counterpart in QUICK.  The variants of class cls (0 .. the class count of qb_class_info
   - 1) for the FP64 or the FP32 kernels: writes up to cap codes, returns how many there are. */
int qb_class_variants(int cls, int fp32, int* codes, int cap);

/* Device form of gpu_upload_cutoff_: the integral and primitive cutoffs, and QUICK's density
   screen cutMatrix(I, J) = max |D| over the shell-pair block (densityCutoff / DNscreen,
   src/schwarz.f90:550-600) computed on the GPU from the device density d_dense (nbasis^2)
   instead of uploaded from the host.  Asynchronous on the library stream. */
int qb_upload_cutoff_device(const double* d_dense, double integralCutoff, double primLimit);

/* Device form of gpu_grad_: adds the two-electron gradient for the device density d_dense to
   d_grad (3 x natom, device), with the cutoffs and density screen last uploaded.  Returns
   when the gradient kernels have finished (their quartet counts are read back). */
int qb_grad_device(const double* d_dense, double* d_grad);

/* Many molecules in one Fock build / gradient (no counterpart in QUICK, which runs one molecule
   per process).  Upload each molecule through the bridge as usual (gpu_setup_ ..
   gpu_upload_cutoff_matrix_), then call qb_batch_add to append its tables; qb_batch_finalize
   sizes the batch's quartet lists for the given cutoffs.  A batched build is one screen launch
   and one launch per angular class for all molecules; quartets pair only bras and kets of the
   same molecule.  Matrices are packed: molecule i's n_i x n_i column-major block at offset
   off_i = sum_{j<i} n_j^2 (qb_batch_layout returns n_i, natom_i and off_i, and the number of
   molecules).  Exchange fraction, mixed split and lane groups are the session's settings at the
   time of the call; the batch keeps its own copies of the tables, so later uploads of other
   molecules do not change it.  qb_batch_reset frees it.  The batch's work matrices are block
   diagonal over the total dimension N = sum n_i (2 N^2 doubles; refused above 120 GB). */
int qb_batch_reset(void);
int qb_batch_add(void);
int qb_batch_finalize(double integralCutoff, double primLimit);
int qb_batch_layout(int* nbasis, int* natom, long long* offsets, int cap);
/* O_out = O_in + G(D) for every molecule (packed device arrays; the density screen is taken
   from D).  Asynchronous on the library stream. */
int qb_batch_fock_device(const double* d_dense, const double* d_o_in, double* d_o_out);
/* d_grad (3 x sum natom_i, molecule after molecule) += the two-electron gradient of every
   molecule at the packed density D.  Asynchronous on the library stream. */
int qb_batch_grad_device(const double* d_dense, double* d_grad);

/* Pulay DIIS coefficients on the device, for an SCF iteration that never waits for the host
   (replaces the host solve of QUICK's electdiis, src/scf.f90:249-523).  d_B: m x m overlaps of
   the stored error vectors (row-major); d_w: m flags, slot i used when d_w[i] != 0 (unused slots
   get c_i = 0); d_newest: the slot of the newest Fock matrix (int64), whose coefficient is 1 if
   the system is singular.  Writes the m coefficients (summing to 1) to d_c.  1 <= m <= 32.
   Asynchronous on the library stream; can be captured into a CUDA graph. */
int qb_diis_solve_device(const double* d_B, const double* d_w, int m, const long long* d_newest, double* d_c);

/* One-electron integrals.  QUICK forms these on the host in Fortran; these entry points follow
   the gpu_* conventions (arguments by pointer, Fortran column-major nbasis^2 matrices) and use
   the uploaded basis, coordinates and charges (gpu_upload_xyz_, gpu_upload_atom_and_chg_,
   gpu_upload_basis_).
   gpu_get1e_: o = H = T + V, the core Hamiltonian of get1e
     (src/quick_one_electron_integral.f90:1699-1809: kinetic part get1eO :1633-1673 with
     dcoeff/aexp, attraction attrashell :1816-1925 / nuclearattra src/nuclear.f90:198-221 with
     gccoeff x cons), full symmetric matrix.
   gpu_get_overlap_: s = S, the overlap matrix of fullx (:31-46).
   qb_oneint_device: both at once into device arrays (either may be null), asynchronous on the
     library stream. */
int gpu_get1e_(double* o);
int gpu_get_overlap_(double* s);
int qb_oneint_device(double* d_S, double* d_H);

/* One-electron and nuclear-repulsion parts of the RHF nuclear gradient (hfgrad,
   src/gradient.f90:49-249): adds to grad (3 x natom, Fortran order) the nuclear repulsion
   term, -2 W dS and 2 D dT over basis-function pairs on different atoms and D dV for the
   nuclear attraction (attrashellopt, src/shell.f90:1747-1830), for the total density D and the
   energy-weighted density W = 2 sum_occ e_k C_k C_k^T (gradient.f90:84-96), both nbasis^2.
   qb_grad1e_device takes device pointers and is asynchronous on the library stream. */
int gpu_grad1e_(double* grad, const double* dense, const double* wdense);
int qb_grad1e_device(const double* d_dense, const double* d_wdense, double* d_grad);

/* Measured FMA throughput of this GPU in GFLOP/s (FP64 if fp64 != 0, else FP32): a
   register-resident FMA chain over 8 blocks per SM, best of 4 timed runs. */
int qb_fma_peak(int fp64, double* gflops);

/* Per angular-momentum class of the last Fock build: the number of primitive quartets that
   passed the primitive screen (cap >= number of classes). */
int qb_count_prim_quartets(long long* per_class, int cap);

/* Number of kernels this library has launched since it was loaded. */
long long qb_launch_count(void);

/* Classes of this build: their (LA, LB, LC, LD) and the shell quartets of the last build. */
int qb_class_info(int* nclasses, int* class_L, long long* class_quartets, int cap);

#ifdef __cplusplus
}
#endif
#endif
