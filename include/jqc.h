/*
 * jqc.h -- C ABI of libjqc.so, the B200 (sm_100a) two-electron engine behind
 * the jax_qc drop-in (jax_examples_b200).
 *
 * Conventions
 *   - Every entry point returns an int status (JQC_OK = 0); on failure
 *     jqc_last_error() returns a message for the calling thread.
 *   - Basis data is passed as HOST arrays; matrices (D, J, K, S, T, V,
 *     gradients, ERI tensors, Boys inputs/outputs) are DEVICE pointers on the
 *     context's device, row-major float64 unless stated.
 *   - `stream` is a cudaStream_t (NULL = legacy default stream).  Entry points
 *     that only launch work on `stream` are asynchronous; the ones that say
 *     "synchronizes" wait for `stream`.
 *   - Layout: basis functions in shell order, Cartesian components of a shell
 *     in libint order (lx descending, then ly descending), as
 *     jax_qc/integrals/mcmurchie_davidson.py:39-50 and overlap.py:58-64.
 *   - A context's device scratch (density block maxima, the compacted work
 *     items of screened builds, gradient force slots) is shared by all calls
 *     on it: calls on one context must be ordered on the GPU (one stream, or
 *     streams ordered by events).  Different contexts are independent.
 */
#ifndef JQC_H_
#define JQC_H_

#ifdef __cplusplus
extern "C" {
#endif

#define JQC_OK 0
#define JQC_ERR_INVALID 1      /* bad argument (maps to ValueError)           */
#define JQC_ERR_CUDA 2         /* CUDA runtime failure                        */
#define JQC_ERR_TOO_LARGE 3    /* output would exceed the size cap            */
#define JQC_ERR_NOT_READY 4    /* call order violated (basis/pairs missing)   */
#define JQC_ERR_UNSUPPORTED 5  /* angular momentum or class not supported     */
#define JQC_ERR_TIMEOUT 6      /* a bounded device wait gave up               */

#define JQC_PREC_FP64 0        /* every quartet in FP64 (the plain kernel)    */
#define JQC_PREC_MIXED 1       /* Q_ij*Q_kl < mixed_tau in FP32, rest FP64    */
#define JQC_PREC_FP32 2        /* every quartet in FP32 (test/diagnostics)    */

typedef struct jqc_ctx jqc_ctx;

/* Message of the last failed call on this thread ("" if none). */
const char *jqc_last_error(void);

/* ABI version (major*100 + minor). */
int jqc_version(void);

/* Create / destroy an engine context bound to CUDA device `device`.
 * Replaces the implicit global state of jax_qc.integrals (integrals/eri.py:69). */
int jqc_ctx_create(int device, jqc_ctx **out);
int jqc_ctx_destroy(jqc_ctx *ctx);

/* Upload a contracted Cartesian basis: shell s has angular momentum l[s]
 * (0..2), nprim[s] primitives starting at prim_off[s] in exps/coefs
 * (coefficients already normalized as jax_qc/basis/normalize.py:91-107 does),
 * centre centres[3s..3s+2] (bohr), atom atom_of_shell[s].  Atoms: n_atom
 * positions atom_xyz[3a..] and nuclear charges atom_charge[a].  cartesian must
 * be 1 (spherical sets are transformed on the host).  Mirrors the BasisSet /
 * Molecule inputs of compute_integrals (integrals/interface.py:26-67). */
int jqc_basis_upload(jqc_ctx *ctx, int n_shell, const int *l, const int *nprim, const int *prim_off,
                     const double *exps, const double *coefs, const double *centres, const int *atom_of_shell,
                     int n_atom, const double *atom_xyz, const double *atom_charge, int cartesian);

/* Build shell-pair data (Gaussian products, E-coefficient inputs) and the
 * Schwarz bounds Q_ij = sqrt(max (ij|ij)) on the device; drop pairs that can
 * never pass Q_ij * max Q >= schwarz_tau, and primitive pairs whose
 * magnitude |K_AB c_a c_b| pi^(5/4) p^(-5/4) is below prim_tau (0 keeps all).
 * Synchronizes `stream`.
 * Replaces integrals/screening.py:32-58 (compute_shell_pair_bounds). */
int jqc_pairs_build(jqc_ctx *ctx, double schwarz_tau, double prim_tau, void *stream);

/* Batch partition: the uploaded atoms (and their shells) belong to n_mol
 * independent molecules, mol_of_atom[a] in 0..n_mol-1.  Shell pairs, quartets,
 * nuclear attraction and gradients then stay inside each molecule, and one
 * jqc_jk / jqc_grad2e / jqc_one_electron call serves all molecules at once
 * over one class-sorted work list (the basis-function matrices are the
 * block-diagonal n x n matrices of the whole batch).  Call after
 * jqc_basis_upload and before jqc_pairs_build; jqc_basis_upload resets it to
 * one molecule.  Replaces the per-molecule loop of geomopt/optimizer.py:55-76
 * (_energy_and_gradient per geometry): a sweep over many geometries or
 * molecules is one call per step instead of one per molecule. */
int jqc_batch_partition(jqc_ctx *ctx, int n_mol, const int *mol_of_atom);

/* Geometry-only update: atom a moves to atom_xyz[3a..3a+2] (bohr) and every
 * shell of atom a with it; exponents, contractions, the batch partition, the
 * molecule mask, launch tuning and the Boys tables stay.  The pair list, work
 * lists and captured graphs are dropped: call jqc_pairs_build before the
 * next J/K, gradient or one-electron call.  Replaces the per-step rebuild of
 * geomopt/optimizer.py:55-76 (_energy_and_gradient builds the basis and all
 * integrals anew for every trial geometry). */
int jqc_set_geometry(jqc_ctx *ctx, const double *atom_xyz);

/* Molecules taking part in the next jqc_pairs_build: active[m] != 0 keeps
 * molecule m of the batch partition, 0 leaves its shell pairs (and so all of
 * its quartets) out of J/K and gradient builds; NULL keeps every molecule.
 * Drops the pair list like jqc_set_geometry.  Serves a geometry sweep whose
 * molecules finish at different steps (geomopt/optimizer.py:130-200 per
 * molecule). */
int jqc_set_molecule_mask(jqc_ctx *ctx, const int *active);

/* Molecule activity read on the device by every later J/K build of a batch
 * context (jqc_batch_partition with more than one molecule), graph replays
 * included: d_active points to n_mol ints in device memory, owned by the
 * caller, who may rewrite them between builds (a converged molecule of a
 * lock-step SCF gets 0).  Each build first compacts the class work lists on
 * the device to the work items holding a task of an active molecule, and the
 * class kernels walk only those (the register kernels as persistent grids
 * over the device-side counts); the J and K blocks of inactive molecules
 * come out zero.  NULL switches it off.  Captured graphs are dropped when the
 * pointer changes.  No reference counterpart (scf/rhf.py:95-169 runs one
 * molecule). */
int jqc_set_molecule_activity(jqc_ctx *ctx, const int *d_active);

/* Counters of the work list for (precision_mode, mixed_tau) as jqc_jk
 * would use it: out[0] shell pairs, out[1] kept pairs, out[2] screened
 * canonical quartets on the FP64 path, out[3] on the FP32 path, out[4]
 * primitive quartets (both), out[5] Cartesian basis functions, out[6] warp
 * tasks, out[7] kernel launches per jqc_jk call.  No reference counterpart
 * (the reference never screens: integrals/screening.py is unused). */
int jqc_stats(jqc_ctx *ctx, int precision_mode, double mixed_tau, long long *out8);

/* Per-class counters: for p in {FP64, FP32 path} and the 21 quartet classes
 * (bra pair class >= ket pair class, pair classes ss ps pp ds dp dd),
 * out[(p*21+q)*3 + 0..2] = canonical quartets, primitive quartets, tasks.
 * No reference counterpart (feeds the FLOP model of the roofline). */
int jqc_class_stats(jqc_ctx *ctx, int precision_mode, double mixed_tau, long long *out126);

/* Schwarz matrix Q (n_shell x n_shell, device) in original shell order.
 * Replaces integrals/screening.py:32-58. */
int jqc_schwarz(jqc_ctx *ctx, double *Q, void *stream);

/* Boys function F_m(T), m = 0..mmax (mmax <= 16) for n values T (device);
 * out is n x (mmax+1), float64 or (fp32 != 0) float32.
 * Replaces integrals/boys.py:34-109 (boys_f0 / boys_fn). */
int jqc_boys(const double *T, long long n, int mmax, void *out, int fp32, void *stream);

/* Primitive Cartesian ERI blocks for n primitive quartets of one class
 * (la lb | lc ld) with la >= lb, lc >= ld, (la,lb) >= (lc,ld): exps is n x 4,
 * centres n x 12 (device); out is n x nc_a nc_b nc_c nc_d.
 * Replaces integrals/obara_saika.py:227-332 (primitive_eri_block). */
int jqc_eri_prim_quartets(int la, int lb, int lc, int ld, long long n, const double *exps, const double *centres,
                          double *out, void *stream);

/* Dense (n,n,n,n) ERI tensor over the kept shell pairs (exact when pairs
 * were built with schwarz_tau = 0).  Fails with JQC_ERR_TOO_LARGE when
 * n^4 * 8 bytes exceeds `max_bytes`.
 * Replaces integrals/eri.py:69-138 (compute_eri_tensor). */
int jqc_eri_tensor(jqc_ctx *ctx, double *out_n4, long long max_bytes, void *stream);

/* One-electron matrices S, T, V (n x n each, device) of the uploaded basis
 * and nuclei.  Replaces integrals/overlap.py:67-85, kinetic.py:42-59 and
 * nuclear.py:62-81 (compute_overlap/kinetic/nuclear_matrix). */
int jqc_one_electron(jqc_ctx *ctx, double *S, double *T, double *V, void *stream);

/* Two-electron part of the nuclear gradient, ADDED into grad (n_atom x 3,
 * device, caller zeroes): grad += 1/2 sum Gamma_abcd d(ab|cd)/dR with
 * Gamma = j_scale D^t_ab D^t_cd - (k_scale/2) sum_s (D^s_ac D^s_bd +
 * D^s_ad D^s_bc), D^t = sum_s D^s over the n_dens densities.  RHF: one total
 * density, j_scale = 1, k_scale = 1/2; UHF: (D_alpha, D_beta), 1, 1.  The
 * derivative integrals are contracted on the fly and never stored.
 * Replaces the finite-difference ERI derivative and its contraction in
 * grad/rhf_grad.py:153-209 (dERI, dJ, dK). */
int jqc_grad2e(jqc_ctx *ctx, int n_dens, const double *D, double j_scale, double k_scale, double *grad,
               void *stream);

/* jqc_grad2e with density screening and per-class timing: quartets whose
 * bound Q_ab Q_cd |Gamma|max is below dens_tau (0 = off) are skipped, with
 * |Gamma|max <= j n^2 m_ab m_cd + (k/2) n (m_ac m_bd + m_ad m_bc) from the
 * per-shell-block density maxima m over the n = n_dens densities.  With
 * class_ms (21 doubles, or NULL) the classes are timed one by one with CUDA
 * events (milliseconds, synchronizes).  No reference counterpart. */
int jqc_grad2e_ex(jqc_ctx *ctx, int n_dens, const double *D, double j_scale, double k_scale, double dens_tau,
                  double *grad, void *stream, double *class_ms);

/* One-electron part of the nuclear gradient, ADDED into grad:
 * grad += sum D_ab d(T+V)_ab/dR - sum W_ab dS_ab/dR (Hellmann-Feynman term of
 * V included); D total density, W energy-weighted density (n x n, device).
 * Replaces the dH/dS finite differences of grad/rhf_grad.py:186-209. */
int jqc_grad1e(jqc_ctx *ctx, const double *D, const double *W, double *grad, void *stream);

/* Direct J/K (the N^4 tensor is never stored): for each of n_dens densities
 * D[d] (n x n, symmetric), J[d] = sum_ls D_ls (mn|ls), K[d] = sum_ls D_ls
 * (ms|ln).  precision_mode as JQC_PREC_*, mixed_tau the FP32/FP64 split on
 * Q_ij*Q_kl, dens_tau the density-weighted skip threshold (0 = off).
 * Replaces scf/fock.py:31-38 (_coulomb / _exchange) and the J/K of
 * build_fock_rhf / build_fock_uhf (fock.py:41-79) and guess.py:87-88. */
int jqc_jk(jqc_ctx *ctx, int n_dens, const double *D, double *J, double *K, int precision_mode, double mixed_tau,
           double dens_tau, void *stream);

/* Allocation-free variant of jqc_jk for callers that cannot allocate device
 * memory when they need a Fock build: a builder called from inside a JAX/XLA
 * program (XLA owns and pre-reserves device memory) or a fixed-memory host
 * loop.  No reference counterpart.  Same arguments and results as jqc_jk with
 * density screening at dens_tau (0 disables it).  Allocates nothing: the
 * work list must already exist (call jqc_jk or jqc_stats once with the same
 * precision_mode/mixed_tau at set-up; otherwise JQC_ERR_NOT_READY), and the
 * density-screening scratch is a static device array of 512*512 floats, so
 * contexts with more than 512 shells get JQC_ERR_TOO_LARGE.  The first call
 * on a device looks the array's address up (cudaGetSymbolAddress); make that
 * first call before any stream capture.  The looked-up address belongs to
 * the device's current primary context: after a cudaDeviceReset in the same
 * process the entry point must not be used again.  All calls share the array
 * and each call rewrites it completely before reading it; calls that overlap
 * on the GPU (different streams or contexts without ordering) race on it. */
int jqc_jk_noalloc(jqc_ctx *ctx, int n_dens, const double *D, double *J, double *K, int precision_mode,
                   double mixed_tau, double dens_tau, void *stream);

/* jqc_jk with the class kernels run one after another on `stream`, each
 * timed with CUDA events; class_ms[p*21+q] receives milliseconds (0 for
 * empty classes).  Synchronizes.  Measurement variant of jqc_jk. */
int jqc_jk_timed(jqc_ctx *ctx, int n_dens, const double *D, double *J, double *K, int precision_mode,
                 double mixed_tau, double dens_tau, void *stream, double *class_ms);

/* CUDA graph capture of any sequence of the stream-ordered calls above
 * (jqc_jk, jqc_grad2e, jqc_grad1e, jqc_one_electron):
 * jqc_graph_begin starts capturing `stream` (a created stream, not the
 * legacy default stream), the calls record their kernels instead of running
 * them, and jqc_graph_end instantiates the graph and returns its id.
 * jqc_graph_launch replays it on a stream with the pointers and settings of
 * the capture (write new densities into the same buffers).  Work lists and
 * scratch must exist before the capture (one ordinary call with the same
 * settings; otherwise the captured call fails with JQC_ERR_NOT_READY).  A
 * new basis, pair list, partition or tuning, or an evicted work list,
 * destroys the context's graphs; their ids then fail with JQC_ERR_INVALID.
 * No reference counterpart (the reference runs the SCF loop eagerly in
 * Python, scf/rhf.py:95-169). */
int jqc_graph_begin(jqc_ctx *ctx, void *stream);
int jqc_graph_end(jqc_ctx *ctx, void *stream, int *graph_id);
int jqc_graph_launch(jqc_ctx *ctx, int graph_id, void *stream);
int jqc_graph_destroy(jqc_ctx *ctx, int graph_id);

/* Launch shape of each of the 21 quartet classes, cfg[4q..4q+3] =
 * threads per block (64/128/256), lane_prims (at most that many primitive
 * quartets per lane and task: the bra primitive pairs of a quartet are split
 * into chunks accordingly), persistent (1: grid capped at the resident
 * blocks, warps stride over the task list) and engine (0: register kernels,
 * lane = ket shell pair, classes with L <= 6; 1: column engine, one warp per
 * quartet, lane = ket Cartesian pair, classes with L >= 5; 2: runtime-class
 * warp engine, every class).  threads and persistent apply to the register
 * kernels only.  A new lane_prims or a change to or from the register engine
 * rebuilds the work lists.  No reference counterpart. */
int jqc_get_tuning(jqc_ctx *ctx, int *cfg84);
int jqc_set_tuning(jqc_ctx *ctx, const int *cfg84);

/* Engine of the ERI-derivative adjoint for one quartet class: 0 register
 * kernels (L <= 4), 1 row engine (bra pair dp or dd; one warp per quartet,
 * lane = bra Cartesian pair), 2 runtime-class warp engine, 3 register
 * kernels with the bra-centre and ket-centre forces in separate block parts
 * (L <= 4; half the per-thread state, R and Boys computed twice).
 * Defaults: row engine for L >= 5, engine 3 for (dp|ss) and (dp|ps),
 * register kernels for the other classes up to L = 4.  No reference
 * counterpart. */
int jqc_set_grad_engine(jqc_ctx *ctx, int quartet_class, int engine);
int jqc_get_grad_engine(jqc_ctx *ctx, int *engines21);

/* Autotuner: times every class of the J/K build for this density, precision
 * and screening (classes serialised, CUDA events, best of two, or one when a
 * build takes over 30 ms) over the engines, then threads (128, 256) x
 * persistent, then lane_prims (64, 128, 256, 512), keeps the fastest
 * shape per class and rebuilds the work list with it.  With cache_path, a
 * line "signature<TAB>84 integers" is appended; a later call whose signature
 * (device, settings, order of magnitude of each class's quartet count)
 * matches a line applies it without timing and sets *from_cache = 1.
 * J and K are overwritten.  Synchronizes.  No reference counterpart. */
int jqc_autotune(jqc_ctx *ctx, int n_dens, const double *D, double *J, double *K, int precision_mode,
                 double mixed_tau, double dens_tau, const char *cache_path, int *from_cache, void *stream);

/* FMA throughput microbenchmark on the current device: `blocks` blocks of
 * 256 threads, each 8 independent FMA chains of 16*iters steps, FP64 or
 * FP32; *tflops = achieved TFLOP/s.  Synchronizes.  No reference
 * counterpart (roofline denominator for the compute-bound kernels). */
int jqc_fp_peak(int fp32, int blocks, int iters, double *tflops, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* JQC_H_ */
