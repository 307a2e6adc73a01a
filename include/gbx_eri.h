/*
 * gbx_eri.h — C ABI of the B200 electron-repulsion-integral engine (libgbx_eri.so).
 *
 * Plain C types only: the caller passes host arrays describing the basis, and device or
 * host pointers for outputs.  Every function returns a status code (GBX_OK = 0); the
 * message of the last failure on the calling thread is available from gbx_last_error().
 *
 * Reference interfaces these entry points replace (paths inside theochem/gbasis):
 *   - gbx_basis_create           <- GeneralizedContractionShell objects handed to
 *                                   ElectronRepulsionIntegral(basis)
 *                                   (gbasis/integrals/electron_repulsion.py:20,
 *                                    gbasis/base.py:32-65, gbasis/contractions.py:118)
 *   - gbx_eri_full / _full_host  <- electron_repulsion_integral(basis, transform=None,
 *                                   notation=...) and BaseFourIndexSymmetric
 *                                   .construct_array_{cartesian,spherical,mix}
 *                                   (gbasis/integrals/electron_repulsion.py:214-281,
 *                                    gbasis/base_four_symm.py:160-557)
 *   - gbx_eri_full with a Schwarz threshold
 *                                <- electron_repulsion_integral_improved(...,
 *                                   schwarz_threshold) (electron_repulsion.py:415-504,
 *                                   gbasis/integrals/_schwarz_screening.py:131-191)
 *   - gbx_schwarz_bounds         <- compute_schwarz_bounds (_schwarz_screening.py:62-90)
 *   - gbx_lincomb                <- construct_array_lincomb's four tensordots
 *                                   (gbasis/base_four_symm.py:559-616)
 *   - gbx_eri_coulomb_j          <- (no direct counterpart: J_ab = sum_cd (ab|cd) D_cd,
 *                                   the contraction gbasis users apply to the tensor)
 *   - gbx_eri_jk                 <- (no direct counterpart: J and K_ac = sum_bd (ab|cd) D_bd
 *                                   from the same tensor)
 *   - gbx_point_charge           <- point_charge_integral / nuclear_electron_attraction_integral
 *                                   (gbasis/integrals/point_charge.py:271-325,
 *                                    nuclear_electron_attraction.py:8-42)
 */
#ifndef GBX_ERI_H
#define GBX_ERI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  GBX_OK = 0,
  GBX_ERR_INVALID = 1,     /* bad argument (shape, value, null pointer) */
  GBX_ERR_UNSUPPORTED = 2, /* angular momentum above the compiled maximum */
  GBX_ERR_OOM = 3,         /* device allocation failed */
  GBX_ERR_CUDA = 4,        /* CUDA runtime / launch error */
  GBX_ERR_TIMEOUT = 5      /* a bounded device wait gave up */
};

/* Output layout of full-tensor calls. */
enum { GBX_CHEMIST = 0, GBX_PHYSICIST = 1 };

typedef struct gbx_basis gbx_basis;

/*
 * Describe a basis of n_shells segmented contractions (one per column of a gbasis
 * coefficient matrix, in basis-function order).  Per shell s:
 *   angmom[s], nprim[s], center[3s..3s+2];
 *   exps / coefs: nprim[s] values each, concatenated over shells (raw contraction
 *     coefficients; primitive normalisation is applied by the engine);
 *   nout[s]: output functions of the shell (L_cart or 2l+1);
 *   sph[s]: 1 if the shell is transformed to real solid harmonics;
 *   pos[10s..]: for each engine-internal component (canonical Cartesian order, or for
 *     spherical shells with l >= 2 the order s_l..s_1, c_0..c_l) the output position
 *     within the shell, or -1;
 *   scl[10s..]: matching scale (norm_cont x component norm or sign).
 * device: CUDA ordinal the basis lives on.
 */
int gbx_basis_create(gbx_basis** out, int n_shells, const int* angmom, const int* nprim,
                     const double* center, const double* exps, const double* coefs,
                     const int* nout, const int* sph, const int8_t* pos, const double* scl,
                     int device);
int gbx_basis_destroy(gbx_basis* b);

/* Two-electron operator of the basis's later integral calls (full tensor, unique integrals, J,
 * J/K): 0 = 1/r, 1 = erf(omega r)/r (long range), 2 = erfc(omega r)/r (short range), the
 * range-separated operators of gbasis/integrals/boys_functions.py:145-223 and
 * get_boys_function (:283-350) that ElectronRepulsionIntegralImproved takes as its boys_func
 * (gbasis/integrals/electron_repulsion.py:284-303).  Schwarz screening keeps the Coulomb
 * bounds, which also bound both attenuated operators (as the reference's screener does). */
int gbx_basis_set_potential(gbx_basis* b, int potential, double omega);
/* Original (generalized-contraction) shell of each segmented shell: Schwarz bounds of a
 * quartet use the bound of the original shell pairs, as gbasis screens whole generalized
 * shells.  Default: every segmented shell is its own group. */
int gbx_basis_set_groups(gbx_basis* b, const int* group);
/* Number of output basis functions N (the tensor is N^4). */
int gbx_basis_nbf(const gbx_basis* b, int64_t* nbf);
/* Unique shell quartets and device bytes the compact store of a full call needs. */
int gbx_basis_stats(const gbx_basis* b, int64_t* n_quartets, int64_t* compact_bytes);

/*
 * Full N^4 float64 tensor into device memory `out` (N^4 doubles, C order).  notation
 * GBX_CHEMIST writes (ab|cd) at out[a,b,c,d]; GBX_PHYSICIST writes <ac|bd> contiguously,
 * i.e. out[a,c,b,d] = (ab|cd).  schwarz_threshold > 0 zeroes shell quartets whose bound
 * Q_ij Q_kl is below it (bounds on blocks without norm_cont, as gbasis's improved path).
 * stream: a cudaStream_t (NULL = legacy default stream).  Asynchronous.
 */
int gbx_eri_full(gbx_basis* b, int notation, double schwarz_threshold, double* out,
                 void* stream);
/*
 * Mixed-precision full tensor (no counterpart in the reference: gbasis computes in FP64
 * only).  With B_q = Schwarz bound of the final values of quartet q (bound on blocks without
 * norm_cont times the largest output scale of each shell): quartets with B_q < skip are
 * zero, those with B_q < fp32 run the vertical/transfer recursions in FP32 (FP64
 * accumulation over primitives, FP64 HRR and transforms), the rest in FP64.
 */
int gbx_eri_full_mixed(gbx_basis* b, int notation, double skip, double fp32, double* out,
                       void* stream);
/* Unique shell quartets only, into the engine's compact store (no N^4 expansion): the
 * integral work of a full call, for bases whose full tensor does not fit in memory.
 * skip = fp32 = 0 is the FP64 form. */
int gbx_eri_unique(gbx_basis* b, double skip, double fp32, void* stream);
/* (ab|cd) in the output functions of the basis for n quadruples idx4[4i..4i+3] = (a,b,c,d),
 * read from the compact store of the last gbx_eri_unique / gbx_eri_full* call on b (the
 * values that call produced, mixed form included) into host memory; synchronous. */
int gbx_unique_values(gbx_basis* b, int64_t n, const int64_t* idx4, double* out_host,
                      void* stream);
/* Device address and length (doubles) of the compact store holding the last call's unique
 * integrals (class blocks of pair functions; NULL / 0 before the first call).  Read-only,
 * valid until the next call on b; for whole-store comparisons such as mixed vs FP64. */
int gbx_compact_view(gbx_basis* b, const double** dev_ptr, int64_t* n_elems);
/* Same as gbx_eri_full, into host memory (page-locked or pageable); synchronous. */
int gbx_eri_full_host(gbx_basis* b, int notation, double schwarz_threshold, double* out_host,
                      void* stream);

/* Schwarz bounds Q_p = sqrt(max |(pp|pp)|) per shell pair of the basis, host array of
 * n_shells*n_shells doubles (symmetric). */
int gbx_schwarz_bounds(gbx_basis* b, double* q_host);

/* 4-index transform: out[i,j,k,l] = sum T[i,a] T[j,b] T[k,c] T[l,d] in[a,b,c,d] on the
 * device (four cuBLAS DGEMMs).  in: N^4, T: n_orb x N (row-major), out: n_orb^4,
 * work: 2 * max(N, n_orb)^4 doubles. */
int gbx_lincomb(const double* in, int64_t n, const double* transform, int64_t n_orb,
                double* out, double* work, void* stream);

/*
 * Allocation-free full tensor (no counterpart in the reference: gbasis has no device code).
 * For callers that cannot call cudaMalloc while they run this library — e.g. a process
 * whose device memory is owned by another allocator that reserved most of the GPU up
 * front, or a pipeline that cannot take the device-wide synchronisation of cudaFree.  Same
 * basis arrays as gbx_basis_create (no handle), same output as gbx_eri_full (device `out`,
 * N^4 doubles, caller-owned), no Schwarz screening.  Every intermediate lives in one static
 * device array of 64 MiB that each GPU loading the library holds until exit; bases needing
 * more are rejected with GBX_ERR_INVALID.  The first call on a device resolves that array's
 * address (cudaGetSymbolAddress) — make it before any stream capture.  Calls share the
 * array: calls that overlap on the GPU race and must be serialised by the caller.
 */
int gbx_eri_full_noalloc(int n_shells, const int* angmom, const int* nprim,
                         const double* center, const double* exps, const double* coefs,
                         const int* nout, const int* sph, const int8_t* pos, const double* scl,
                         int notation, double* out, void* stream);

/*
 * Batched full tensors of many molecules (no counterpart in the reference: gbasis computes
 * one basis per electron_repulsion_integral call; this replaces a Python loop of such calls).
 * The molecules' shells are given back to back in the gbx_basis_create arrays, molecule m
 * owning mol_nshells[m] consecutive shells.  gbx_batch_run writes molecule m's N_m^4 float64
 * tensor to the device buffer outs[m] (host array of n_mol device pointers); the first run
 * captures all launches — one class kernel per block type for the whole batch, then one
 * batched expansion — into a CUDA graph that later runs replay (with any outputs and
 * notation).  Ordered after prior work on `stream` and before later work on it.
 */
typedef struct gbx_batch gbx_batch;
int gbx_batch_create(gbx_batch** out, int n_mol, const int* mol_nshells, const int* angmom,
                     const int* nprim, const double* center, const double* exps,
                     const double* coefs, const int* nout, const int* sph, const int8_t* pos,
                     const double* scl, int device);
int gbx_batch_destroy(gbx_batch* b);
/* nbf: n_mol entries (may be NULL); total unique shell quartets; compact store bytes. */
int gbx_batch_info(const gbx_batch* b, int64_t* nbf, int64_t* n_quartets,
                   int64_t* compact_bytes);
int gbx_batch_run(gbx_batch* b, int notation, double* const* outs, void* stream);
/* 1 (default): replay a captured CUDA graph; 0: launch eagerly every run. */
int gbx_batch_set_graph(gbx_batch* b, int on);
/* 1: the FP64 run's class kernels become ONE persistent launch (a multi-class work queue:
 * every block type's quartets, largest types first, drawn by warps from a single counter and
 * evaluated by the class's recursion programs), followed by the batched expansion, captured
 * and replayed as above; 0 (default): one class kernel per block type.  The mixed form and
 * per-type profiling always use the per-type kernels.  Changing it drops the captured graph.
 * No counterpart in the reference (a Python loop of per-molecule calls). */
int gbx_batch_set_queue(gbx_batch* b, int on);
/* Block types of a batch (one class kernel launch each) and their team of lanes per quartet
 * (register kernel; the autotuner's knob).  Setting a team drops the captured graph.  With
 * profiling on, runs launch the types one after another (no graph) and gbx_batch_type_times
 * returns each type's kernel time (ms) of the last run. */
int gbx_batch_num_types(const gbx_batch* b, int* n);
int gbx_batch_type_info(const gbx_batch* b, int k, int* cls4, int* team, double* avg_prims,
                        int64_t* n_quartets);
int gbx_batch_set_team(gbx_batch* b, int k, int team);
/* The same knobs per block type of a batch (changing them drops the captured graph). */
int gbx_batch_set_type_config(gbx_batch* b, int k, int variant, int ctas_per_sm);
int gbx_batch_set_profiling(gbx_batch* b, int on);
int gbx_batch_type_times(gbx_batch* b, double* ms, int n);
/* Mixed-precision form of gbx_batch_run (the batched counterpart of gbx_eri_full_mixed; no
 * counterpart in the reference, which has neither batches nor a mixed form): quartets whose
 * final-value bound Q_p Q_q is below `skip` are zero, those below `fp32` in light classes run
 * their recursions in FP32.  The bounds are computed once per batch (first mixed run; make it
 * before any stream capture), the lists once per pair of thresholds; the mixed launches are
 * captured into their own CUDA graph.  gbx_batch_mixed_counts: quartets of the last lists in
 * FP64, in FP32 and left out (all 0 before the first mixed run). */
int gbx_batch_run_mixed(gbx_batch* b, int notation, double skip, double fp32,
                        double* const* outs, void* stream);
int gbx_batch_mixed_counts(const gbx_batch* b, int64_t* n_fp64, int64_t* n_fp32,
                           int64_t* n_skipped);

/* Coulomb matrix J[a,b] = sum_cd (ab|cd) D[c,d] from the screened unique quartets
 * (full tensor never stored; only quartets with Q_p Q_q >= schwarz_threshold are enumerated,
 * Q the bounds of compute_schwarz_bounds).  D, J: device N x N row-major (D symmetric).
 * gbx_last_counts: quartets computed and screened out. */
int gbx_eri_coulomb_j(gbx_basis* b, const double* D, double schwarz_threshold, double* J,
                      void* stream);

/* Mixed-precision direct Coulomb matrix: quartets whose final-value bound (Q_p Q_q over the
 * output functions, norm_cont and transforms included) is below `skip` are left out, those
 * below `fp32` in light classes run their recursions in FP32, the rest in FP64; the
 * contraction with D and J stay FP64.  0 < skip <= fp32 < 1.  Same replacement as
 * gbx_eri_coulomb_j (no direct counterpart in gbasis). */
int gbx_eri_coulomb_j_mixed(gbx_basis* b, const double* D, double skip, double fp32, double* J,
                            void* stream);

/* Coulomb and exchange matrices of a density D (any N x N, not only symmetric):
 *   J[a,b] = sum_cd (ab|cd) D[c,d],   K[a,c] = sum_bd (ab|cd) D[b,d]   (chemist notation),
 * from the unique integrals of the screened quartets (the N^4 tensor is never formed; the
 * unique-integral store, N^4/8 values, is).  No gbasis counterpart: gbasis users contract the
 * tensor of electron_repulsion_integral (gbasis/integrals/electron_repulsion.py:214-281) this
 * way.  D, J, K: device N x N row-major, three different buffers. */
int gbx_eri_jk(gbx_basis* b, const double* D, double schwarz_threshold, double* J, double* K,
               void* stream);

/* Device-side counters of the last call on this basis: quartets computed and screened. */
int gbx_last_counts(const gbx_basis* b, int64_t* computed, int64_t* screened);

/* Quartets of the last compact-store call on this basis (full tensor or unique integrals) by
 * treatment: computed in FP64, computed with FP32 recursions (mixed form), and left out (their
 * integrals are zero: below the mixed form's skip bound, or screened).  No counterpart in the
 * reference: gbasis computes every quartet in FP64. */
int gbx_mixed_counts(const gbx_basis* b, int64_t* n_fp64, int64_t* n_fp32, int64_t* n_left_out);

/* Mixed form: a class block's FP32 quartets get their own FP32 launch only when they number at
 * least min_quartets and at least 1/share of the block; otherwise they stay in its FP64 list
 * (default 65536 and 4: smaller lists cost more in launch, table staging and tail than FP32
 * saves).  No counterpart in the reference. */
int gbx_basis_set_fp32_lists(gbx_basis* b, int64_t min_quartets, int64_t share);

/* Phase timing: level 1 records CUDA events on the call's stream around the work-list
 * build, the class kernels and the expansion (gbx_phase_times waits for the last call and
 * returns the three durations in ms); level 2 also times every class block, running them
 * one after another on the call's stream instead of concurrently; 0 turns it off. */
int gbx_set_profiling(gbx_basis* b, int on);
int gbx_phase_times(gbx_basis* b, double* ms3);

/* Work decomposition per class block (the autotuner's knobs): a class block is the set of
 * quartets of one (bra pair class, ket pair class); `team` is how many lanes share one
 * quartet's primitive loop in the register kernel (power of two, 1..32); n_quartets is the
 * block's unique quartets (after a direct-J call: the quartets that call computed).  With
 * profiling on, gbx_block_times returns each block's kernel time of the last call (ms); level 2
 * also times the blocks of a direct-J call. */
int gbx_num_blocks(const gbx_basis* b, int* n);
int gbx_block_info(const gbx_basis* b, int k, int* cls4, int* team, double* avg_prims,
                   int64_t* n_quartets);
int gbx_set_team(gbx_basis* b, int k, int team);
/* Further launch knobs of block k (the autotuner's): variant 0 runs a heavy class that has
 * both kernels on the split register kernel, 1 on the line kernel; for the classes whose line
 * kernel has the interpreted tail, 0 picks between the one-warp-per-quartet line kernel and
 * its group form (a CTA of 4 warps per quartet) by the warps the former keeps resident, 1
 * forces the former and 2 the group form (no effect on other classes); ctas_per_sm (1..32)
 * caps the register kernel's grid at that many CTAs per SM.
 * gbx_basis_set_streams: number of concurrent streams (1..16, default 6) the class blocks of
 * a call are spread over.  No reference counterpart (gbasis runs one quartet at a time). */
int gbx_set_block_config(gbx_basis* b, int k, int variant, int ctas_per_sm);
int gbx_basis_set_streams(gbx_basis* b, int n_streams);
int gbx_block_times(gbx_basis* b, double* ms, int n);

/* Point-charge interaction integrals of the basis's functions (the replacement of
 * point_charge_integral, gbasis/integrals/point_charge.py:271-325, and with sum_points = 1 of
 * nuclear_electron_attraction_integral, gbasis/integrals/nuclear_electron_attraction.py:8-42):
 *   sum_points = 0: out[(a*N + b)*n_points + c] = -charges[c] (a| 1/|r - R_c| |b)
 *   sum_points = 1: out[a*N + b] = sum_c -charges[c] (a| 1/|r - R_c| |b)
 * coords: host n_points x 3, charges: host n_points (finite); out: device, row-major.  The call
 * returns once the kernels are done (it synchronizes `stream`). */
int gbx_point_charge(gbx_basis* b, int n_points, const double* coords, const double* charges,
                     int sum_points, double* out, void* stream);

/* Device memory that destroyed bases gave back is kept (up to 2 GiB per device) for the next
 * basis of the process: the full-tensor call of the Python layer (the replacement of
 * gbasis/integrals/electron_repulsion.py:214-281, which allocates per call) builds and drops a
 * basis every time.  This frees that cache on every device. */
int gbx_release_cached_memory(void);

/* Copy of the last error message on this thread (NUL-terminated, truncated to len). */
int gbx_last_error(char* buf, size_t len);

/* *on = 1 in the bounds-checking build (libgbx_eri_debug.so, compiled with
 * GBX_DEBUG_BOUNDS=1), else 0.  In that build every kernel store into the compact store, the
 * work lists, the N^4 tensor (or a host-copy slab) and J / K, and every compact-store read
 * of the expansions, is index-checked; a call whose kernels went out of range waits for its
 * stream and returns GBX_ERR_INVALID naming the site and the index, instead of writing there.
 * It stands in for a device memory checker.  No counterpart in the reference. */
int gbx_debug_bounds(int* on);

/* Sustained FP64 FMA rate of the device (TFLOP/s) from a dependent-FMA microbenchmark. */
int gbx_fp64_peak(int device, double* tflops);

/* Measured rate (TFLOP/s) of one arithmetic pipe of the device: pipe 0 = FP64 FMA (as
 * gbx_fp64_peak), 1 = FP64 tensor-core mma.sync m8n8k4, 2 = FP32 FMA.  The roofline
 * denominators of the FP64 and FP32 recursions, and the evidence for or against FP64 tensor
 * cores for the small dense contractions (HRR, spherical transform).  No reference
 * counterpart (gbasis has no device code). */
int gbx_pipe_peak(int device, int pipe, double* tflops);

/* Boys values F_0..F_{m_max}(T[i]) on the current device, computed by the same device
 * function the class kernels use (Taylor table for T < 40, asymptotic form above), for
 * checking that function on its own.  Replaces, for that purpose,
 * boys_function_standard / boys_function_recursion (gbasis/integrals/boys_functions.py:26-63,
 * :102-142).  T: host, n finite values >= 0 (anything else is GBX_ERR_INVALID); F: host,
 * n x (m_max + 1) row-major; 0 <= m_max <= 13.  Synchronous. */
int gbx_boys_eval(int m_max, int64_t n, const double* T, double* F);

#ifdef __cplusplus
}
#endif
#endif /* GBX_ERI_H */
