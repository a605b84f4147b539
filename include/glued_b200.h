/*
 * glued_b200.h — C ABI of the B200-native GLUED hot path.
 *
 * The library replaces the device side of GLUED's CalcGluedForceKernel (CV
 * evaluation -> MetaD/OPES bias -> chain-rule force scatter into OpenMM's 2^32
 * fixed-point force buffer) with hand-written sm_100a CUDA kernels, behind the
 * same descriptor (GluedForce) and kernel (CalcGluedForceKernel) interfaces.
 * Reference citations are relative to the GLUED source tree.
 *
 * Conventions
 *   - Every function returns 0 on success or a negative GLUED_E_* code; the
 *     message of the last failure on the calling thread is glued_last_error().
 *     No C++ exception crosses this boundary (the reference throws
 *     OpenMMException for the same conditions: openmmapi/src/GluedForce.cpp:48-99,
 *     platforms/common/src/CommonGluedKernels.cpp:3886-3927,
 *     platforms/common/src/CommonSerialization.cpp:187-236).
 *   - Caller owns every host buffer and the bound device buffers (posq, atom
 *     index, force buffer). Handles own their device state.
 *   - Device work is enqueued on the bound stream; only the calls documented as
 *     "synchronizing" wait for the device.
 *   - Positions: OpenMM posq layout, float4 per GPU slot (x, y, z, charge), in nm.
 *     Force buffer: int64[3 * padded_num_atoms], field-major, value * 2^32,
 *     accumulated with += (OpenMM's long force buffer).
 */
#ifndef GLUED_B200_H
#define GLUED_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GLUED_OK 0
#define GLUED_E_INVALID (-1)    /* bad argument / spec validation failure */
#define GLUED_E_CUDA (-2)       /* CUDA runtime error */
#define GLUED_E_STATE (-3)      /* call not valid in the current state */
#define GLUED_E_CORRUPT (-4)    /* corrupt / mismatched bias-state blob */
#define GLUED_E_UNSUPPORTED (-5)/* CV or bias type outside this build's scope */

typedef struct glued_force glued_force;     /* GluedForce descriptor */
typedef struct glued_context glued_context; /* per-Context kernel state */
typedef struct glued_batch glued_batch;     /* many walkers, one graph of two launches per step */

/* Message of the last failed call on this thread ("" if none). */
const char* glued_last_error(void);
/* Library version string. */
const char* glued_version(void);

/* ------------------------------------------------------------------ descriptor
 * GluedForce (openmmapi/include/GluedForce.h:113-239,
 * openmmapi/src/GluedForce.cpp:11-133). Type codes are the reference's
 * CVType/BiasType enums (GluedForce.h:27-95).                                  */
int glued_force_create(glued_force** out);
int glued_force_copy(const glued_force* src, glued_force** out);      /* GluedForce.cpp:16-26 */
int glued_force_destroy(glued_force* f);
/* addCollectiveVariable (GluedForce.cpp:44-61): *out_index = first CV value slot. */
int glued_force_add_cv(glued_force* f, int type, const int* atoms, int n_atoms,
                       const double* params, int n_params, int* out_index);
/* addBias (GluedForce.cpp:81-105): rejects CV indices outside [0, numCVValues). */
int glued_force_add_bias(glued_force* f, int type, const int* cv_indices, int n_cvs,
                         const double* params, int n_params, const int* int_params,
                         int n_int_params, int* out_index);
/* addExpressionCV / addPyTorchCV (GluedForce.cpp:164-203): stored and serialized;
 * a context built from a force holding them reports GLUED_E_UNSUPPORTED.       */
int glued_force_add_expression_cv(glued_force* f, const char* expression, const int* inputs,
                                  int n_inputs, int* out_index);
int glued_force_add_pytorch_cv(glued_force* f, const char* model_path, const int* atoms,
                               int n_atoms, const double* params, int n_params, int* out_index);
int glued_force_num_cv_values(const glued_force* f, int* out);        /* getNumCollectiveVariables */
int glued_force_num_cv_specs(const glued_force* f, int* out);         /* getNumCollectiveVariableSpecs */
int glued_force_num_biases(const glued_force* f, int* out);
/* getCollectiveVariableInfo (GluedForce.cpp:67-76). Two-call protocol: pass
 * NULL buffers to read the sizes into *n_atoms / *n_params.                     */
int glued_force_get_cv(const glued_force* f, int idx, int* type, int* atoms, int* n_atoms,
                       double* params, int* n_params);
/* getExpressionCVInfo / getPyTorchCVModelPath: *len in/out, bytes incl. NUL.   */
int glued_force_get_cv_string(const glued_force* f, int idx, char* buf, size_t* len);
/* getBiasInfo (GluedForce.cpp:111-121), same two-call protocol.                 */
int glued_force_get_bias(const glued_force* f, int idx, int* type, int* cvs, int* n_cvs,
                         double* params, int* n_params, int* int_params, int* n_int_params);
int glued_force_set_temperature(glued_force* f, double kelvin);
int glued_force_get_temperature(const glued_force* f, double* kelvin);
int glued_force_set_pbc(glued_force* f, int yes);
int glued_force_get_pbc(const glued_force* f, int* yes);
int glued_force_set_force_group(glued_force* f, int group);
int glued_force_get_force_group(const glued_force* f, int* group);
/* Test-only hooks (GluedForce.h:181-193): constant/per-atom/PBC test forces and
 * injected dU/dCV that bypass the bias kernels.                                 */
int glued_force_set_test_force(glued_force* f, int mode, double scale);
int glued_force_get_test_force(const glued_force* f, int* mode, double* scale);
int glued_force_set_test_bias_gradients(glued_force* f, const double* g, int n);
int glued_force_get_test_bias_gradients(const glued_force* f, double* g, int* n);
/* XML in OpenMM's XmlSerializer layout for GluedForceProxy
 * (serialization/src/GluedForceProxy.cpp:15-138). *len in/out incl. NUL.       */
int glued_force_serialize_xml(const glued_force* f, char* buf, size_t* len);
int glued_force_deserialize_xml(const char* xml, glued_force** out);

/* --------------------------------------------------------------------- context
 * CalcGluedForceKernel (openmmapi/include/GluedKernels.h:23-105) as implemented
 * by CommonCalcGluedForceKernel (platforms/common/src/CommonGluedKernels.cpp:
 * 4608-5288). One context per OpenMM Context on one GPU.                       */
/* initialize(System, GluedForce) (CommonGluedKernels.cpp:4608-4644): validates the
 * specs, flattens them and allocates device state on the current device.
 * masses: double[num_particles] (System::getParticleMass), may be NULL = 1.0.   */
int glued_context_create(const glued_force* f, int num_particles, const double* masses,
                         glued_context** out);
int glued_context_destroy(glued_context* c);
/* Bind OpenMM's device buffers (ComputeContext::getPosq / getAtomIndexArray /
 * getLongForceBuffer / getPaddedNumAtoms) and the stream to enqueue on.
 * atom_index: int[num_particles], GPU slot -> user atom; NULL = identity.       */
int glued_context_bind(glued_context* c, void* stream, const void* posq, const int* atom_index,
                       long long* force_buffer, int padded_num_atoms);
/* OpenMM reordered atoms (ComputeContext::getAtomsWereReordered): rebuild the
 * user -> GPU slot map on the device (CommonCVKernels.cpp:113-320).             */
int glued_context_atoms_reordered(glued_context* c);
/* Periodic box vectors a, b, c (reduced form, nm), row-major double[9].        */
int glued_context_set_box(glued_context* c, const double box[9]);
/* Current step count, for callers that evaluate outside updateState.           */
int glued_context_set_step(glued_context* c, long long step);
/* execute(ContextImpl&, includeForces, includeEnergy) (CommonGluedKernels.cpp:
 * 4646-5048). With include_energy, synchronizing; *energy_out = total bias.     */
int glued_context_execute(glued_context* c, int include_forces, int include_energy,
                          double* energy_out);
/* updateState(ContextImpl&, step) (CommonGluedKernels.cpp:5050-5157): pace-gated
 * deposition from the previous execute()'s CVs; once per step.                  */
int glued_context_update_state(glued_context* c, int step);
/* downloadCVValues / getCurrentCVs (CommonGluedKernels.cpp:5264-5271); synchronizing. */
int glued_context_get_cv_values(glued_context* c, double* out, int n);
/* downloadLastBias (CommonGluedKernels.cpp:5273-5287); synchronizing.           */
int glued_context_get_last_bias(glued_context* c, double* out);
/* getBiasStateBytes / setBiasStateBytes: 'GPUS' v1 blob
 * (platforms/common/src/CommonSerialization.cpp:20-411). *len in/out.          */
int glued_context_get_bias_state(glued_context* c, char* buf, size_t* len);
int glued_context_set_bias_state(glued_context* c, const char* buf, size_t len);
/* getOPESMetrics (CommonGluedKernels.cpp:5164-5210): out = [zed, rct, nker, neff]. */
int glued_context_opes_metrics(glued_context* c, int opes_index, double out[4]);
/* getKernelSigmas (CommonGluedKernels.cpp:5212-5232); *n in/out floats.         */
int glued_context_kernel_sigmas(glued_context* c, int opes_index, float* out, int* n);
/* getMultiWalkerPtrs / redirectToPrimaryBias (platforms/cuda/src/
 * CudaGluedKernelFactory.cpp:30-46, CommonGluedKernels.cpp:5234-5262). bias_index
 * is the global addBias index. METAD: [grid]; OPES: [centers, sigmas, logW,
 * numKernels, numAllocated]. *n in/out.                                         */
int glued_context_multiwalker_ptrs(glued_context* c, int bias_index, long long* out, int* n);
int glued_context_set_multiwalker_ptrs(glued_context* c, int bias_index, const long long* ptrs, int n);
/* Device pointers of the per-step outputs (for zero-copy consumers such as the
 * autograd path): cvValues double[numCV], cvBiasGradients double[numCV],
 * Jacobian rows (atom int, gx/gy/gz float, cv int)[num_rows].                   */
int glued_context_device_arrays(glued_context* c, void** cv_values, void** dudcv, void** jac_atom,
                                void** jac_gx, void** jac_gy, void** jac_gz, void** jac_cv,
                                int* num_cvs, int* num_rows);
/* Measurement hooks (no reference counterpart). profile_phases times each launch
 * group of execute() separately with CUDA events on the bound stream, reps
 * launches each: out[i] = mean ms of phase i in the order simple CVs, group CVs,
 * coordination pairs, coordination finalize, biases, scatter (*n in/out).
 * launch_count = kernels this context enqueued so far (graph replays count
 * their kernel nodes).                                                        */
int glued_context_profile_phases(glued_context* c, int reps, double* out, int* n);
int glued_context_launch_count(glued_context* c, long long* count);
/* FP32 FMA throughput of the current device in TFLOP/s (FMA = 2 flops),
 * measured with a register-resident FMA-chain kernel (synchronizing).         */
int glued_measure_fp32_peak(double* tflops);
/* Hill-slice staging probe (synchronizing): ctas CTAs each copy an equal slice of
 * the three float arrays of a num_hills table into shared memory, timed alone
 * after an L2 flush, reps launches per form: out[0] = us per launch with 16-byte
 * cp.async copies, out[1] = with one bulk copy (cp.async.bulk, mbarrier
 * completion, no multicast) per array; *status bit 0: a bulk wait gave up.     */
int glued_measure_hill_staging(int num_hills, int ctas, int reps, double out[2], int* status);
/* Test hook: index of the last OPES deposit decision of OPES bias opes_index
 * (>= 0 merged into that kernel, -1 appended, -2 warm-up skip, -3 table full).  */
int glued_context_opes_last_decision(glued_context* c, int opes_index, int* decision);
/* Sum precision (no reference counterpart; the reference sums in FP32/FP64 as
 * its kernels are written). kernel_sums, for the OPES and hill-sum MetaD kernel
 * sums: 0 = FP64 evaluation and sums (default), 1 = FP32 Gaussians and plain FP32
 * sums, 2 = FP32 Gaussians and two-sum compensated FP32 sums; in modes 1 and 2
 * OPES heights are exp(logW - M) with M the largest logW of a warp, rescaled by
 * exp(M) in FP64, and the hill truncation exponent is formed in FP64.
 * coordination: 0 = per-lane FP32 A-gradient sums over a whole tile run (default),
 * 1 = blocked, flushed into the exact 64-bit fixed-point sums every 8 steps
 * (<= 32 pairs per FP32 partial). Takes effect at the next execute.            */
int glued_context_set_sum_precision(glued_context* c, int kernel_sums, int coordination);
/* Pair list of a cutoff coordination CV (CV_COORDINATION_CUTOFF on the default
 * cell-list path; params[4] = 1 selects all-pairs tiles instead and has no list)
 * at the bound positions and box: pairs (a, b) of group-A index a and group-B
 * index b with 1e-20 <= r^2 < rc^2 (r^2 in FP64 from the FP32 positions,
 * minimum image floor(d / L + 1/2)), sorted; *n = number of pairs, min(cap, *n)
 * pairs (2 ints each) copied to out (may be NULL when cap is 0). cv_index is
 * the CV's value index. Synchronizing. No reference counterpart.              */
int glued_context_coordination_pairs(glued_context* c, int cv_index, int* out, long long cap, long long* n);
int glued_context_get_sum_precision(glued_context* c, int* kernel_sums, int* coordination);

/* ------------------------------------------------------ differentiable bias
 * Contact map + path CV + hill bias E(CMAP, s) with a hand-written backward
 * (no reference counterpart: GLUED has no autograd path; the CVs are its contact
 * map, CommonGluedKernels.cpp:1236-1323, and path CV, :641-794). dtype 0 = FP32,
 * 1 = FP64 for every R-typed array. All arrays are device memory owned by the
 * caller. out: double[7 + F] = E, CMAP, s, z, S, w_0..w_{F-1}, dE/dCMAP, dE/ds.
 * partials: double[n_partials] (CMAP partial sums, one per CTA of the forward).
 * backward: grad_energy = device double dL/dE; acc = int64[3 * n_atoms] scratch
 * (2^40 fixed point); outputs dL/d(positions, r0, frames, heights).           */
typedef struct glued_ad_spec {
    const void* pos;        /* R[n_atoms][3] */
    int nAtoms;
    const int* pairs;       /* int[P][2] */
    int nPairs;
    const void* r0;         /* R[P] */
    const float* nmw;       /* float[P][3]: n, m, w (integer n, m) */
    const int* pathAtoms;   /* int[M] */
    int M;
    const void* frames;     /* R[F][M][3] */
    int F;                  /* <= 128 */
    double lambda;
    const double* hillC;    /* double[K][2]: (CMAP, s) centres */
    const void* heights;    /* R[K] */
    int K;
    double sig[2];
    int periodic;
    double box[3];          /* rectangular box lengths when periodic */
} glued_ad_spec;
int glued_ad_forward(int dtype, void* stream, const glued_ad_spec* spec, double* out, double* partials,
                     int n_partials);
int glued_ad_backward(int dtype, void* stream, const glued_ad_spec* spec, const double* out,
                      const double* grad_energy, long long* acc, void* grad_pos, void* grad_r0, void* grad_frames,
                      void* grad_heights);

/* ------------------------------------------------------ no-allocation variant
 * No counterpart in the reference. For callers that cannot allocate device
 * memory while they evaluate forces (an engine that reserves all device memory
 * at start-up and forbids cudaMalloc in its step loop, or that manages the
 * device heap with its own allocator): one coordination CV evaluated with its
 * tile partials in a fixed array that is part of this library's device image,
 * GLUED_NOALLOC_SCRATCH_BYTES (4 MiB) per GPU, resident on every GPU that
 * loads the library until the process exits. The call allocates nothing:
 * no cudaMalloc, no cudaFree, no allocating library routine.
 *   posq       float4[...] device positions (slot order)
 *   group_a/b  int device arrays of slot indices, n_a and n_b entries
 *   r0, n, m   rational switch (1 - (r/r0)^n) / (1 - (r/r0)^m), no cutoff;
 *              r0, n and m must be finite and > 0 (else GLUED_E_INVALID);
 *              n == m gives the constant switch 1. Integer n, m <= 64 are
 *              evaluated as S_n(x)/S_m(x) in FP32, other exponents with the
 *              reference formula in FP64, as the context path does; CN and
 *              dCN/dx agree with glued_context_execute to FP32 partial-sum
 *              rounding (measured: CN within 1e-7 relative, gradients within
 *              9e-6 of the largest one, for 6/12, 8/14 and 6.5/11)
 *   periodic   minimum image in box[9] (a, b, c; host array) when non-zero
 *   cn_out     device double[1]: the coordination number
 *   grad_out   device float[3 * (n_a + n_b)]: dCN/dx, component-major
 *              (x of all rows, then y, then z), rows = group A then group B
 * Sizes whose partials exceed the array are rejected with GLUED_E_INVALID
 * (about 2,048 x 8,192 atoms fit). Every call looks up the array's device
 * address in the current context (this allocates nothing, and stays valid
 * across a cudaDeviceReset); the first call on a device may load the module:
 * make it before any stream capture. Every call shares the one array and leaves its contents
 * behind; nothing in it needs to start at zero. Calls whose work overlaps on
 * the GPU (different streams, or a second call before the first finished on
 * another stream) race on the array and corrupt each other's results.     */
#define GLUED_NOALLOC_SCRATCH_BYTES 4194304
int glued_coordination_noalloc(void* stream, const void* posq, const int* group_a, int n_a, const int* group_b,
                               int n_b, double r0, double n, double m, int periodic, const double box[9],
                               double* cn_out, float* grad_out);

/* ----------------------------------------------------------------------- batch
 * Many walkers on one GPU evaluated by one graph per step (a persistent
 * kernel for the coordination pairs, then a finalize kernel that also sums the
 * shared hill table per walker)
 * (no reference counterpart as a kernel: it replaces the reference's
 * one-Context-per-walker stepping, tests/test_multiwalker.py:156-158, and its
 * shared-bias pointer aliasing, CommonGluedKernels.cpp:5234-5262).
 * Scope: distance, angle, dihedral and coordination CVs; HARMONIC biases per
 * walker; at most one METAD_HILLS bias (<= 2 CVs, on distance/angle/dihedral
 * CVs) whose hill table is shared by all walkers (parameters of walker 0). */
typedef struct glued_walker_desc {
    const void* posq;          /* float4[padded] device; slot order = user atom order */
    long long* force_buffer;   /* int64[3 * padded] device, += 2^32 fixed point */
    int num_atoms;
    int padded_num_atoms;
    double box[9];             /* a, b, c (nm) */
} glued_walker_desc;

/* forces[w] describes walker w. Every walker must have the same CV and bias
 * structure (types, order, coordination group sizes); atoms and parameters may
 * differ per walker. The descriptors are copied.                               */
int glued_batch_create(const glued_force* const* forces, int num_walkers, const glued_walker_desc* walkers,
                       glued_batch** out);
int glued_batch_destroy(glued_batch* b);
int glued_batch_set_stream(glued_batch* b, void* stream);
/* Tuning: tune[4] = {ra (A atoms per warp of a coordination tile: 4 or 8, tile =
 * 16 ra atoms), finalize_parts (finalize CTAs per walker, 512 coordination
 * rows at most per CTA; 0 = the fewest: one when the walker has at most 512
 * rows, otherwise the CTAs that cover them plus one that completes the walker;
 * raised to that number when lower), finalize launch (0: a programmatic
 * dependent launch of the runs kernel, 1: a plain stream-ordered launch), B chunk
 * (128 or 256 atoms; 0 = 128)}. Tile shapes other than ra 8 / chunk 128 exist for
 * the n = 6, m = 12 switch in rectangular or no boxes with plain FP32 sums.
 * autotune times every available shape x finalize parts x launch mode on the
 * live walkers, each timed step after an L2 flush (forces of the trial launches
 * go to a scratch buffer; a 192 MB flush buffer is allocated for the call and
 * freed), keeps the fastest and returns it in tune (synchronizing). The choice
 * is cached for the process per (walker count, coordination group sizes, hill
 * count to a power of two, box kind, switch kind, sum precision);
 * glued_batch_autotune uses the cache, glued_batch_autotune_ex(use_cache = 0)
 * times again (*cached = 1 when the returned choice came from the cache).
 * glued_batch_get_tuning returns the tuning in effect (finalize_parts as
 * launched).                                                                   */
int glued_batch_set_tuning(glued_batch* b, const int tune[4]);
int glued_batch_get_tuning(glued_batch* b, int tune[4]);
int glued_batch_autotune(glued_batch* b, int tune[4]);
int glued_batch_autotune_ex(glued_batch* b, int use_cache, int tune[4], int* cached);
/* Sum precision of the batch: 1 = plain FP32 hill and coordination sums
 * (default), 2 = two-sum compensated FP32 hill sums (per lane and through the
 * lane tree, hi + lo in FP64 per runs CTA) and blocked coordination A sums
 * (as glued_context_set_sum_precision coordination = 1).                       */
int glued_batch_set_sum_precision(glued_batch* b, int mode);
int glued_batch_get_sum_precision(glued_batch* b, int* mode);
/* One step for all walkers: CVs, biases and force scatter (one graph of two
 * launches: the coordination/hill runs kernel, then the finalize kernel).
 * Forces are added to each walker's buffer.                                    */
int glued_batch_execute(glued_batch* b);
/* Deposition at pace (once per step, after the step's first execute): one hill
 * per walker, walker order.                                                    */
int glued_batch_update_state(glued_batch* b, int step);
/* energies: double[num_walkers]; cv_values: double[num_walkers * num_cvs].     */
int glued_batch_get_energies(glued_batch* b, double* energies);
int glued_batch_get_cv_values(glued_batch* b, double* cv_values);
int glued_batch_num_cvs(glued_batch* b, int* n);
/* Shared hill table: count, load (replace) and read back (centres n*D, heights n). */
int glued_batch_num_hills(glued_batch* b, int* n);
int glued_batch_set_hills(glued_batch* b, const double* centers, const double* heights, int n);
int glued_batch_get_hills(glued_batch* b, double* centers, double* heights, int n);
/* Status word of the batch's device checks (0 = ok; bit 0: a deposit found the
 * hill table full, maxHills, and dropped hills). Sticky until the batch is
 * destroyed.                                                                   */
int glued_batch_status(glued_batch* b, int* status);
int glued_batch_launch_count(glued_batch* b, long long* count);
/* Profiling: runs one regular step (forces are accumulated as by execute), as
 * the step graph launches it, between two CUDA events, every CTA time-stamped,
 * then a second step with each launch between CUDA events (forces accumulated
 * again). out[28], times in microseconds: {the step (events); last finalize CTA end
 * after the first runs CTA started; staging prologue of a runs CTA (median,
 * max); end of a CTA's coordination steps after the first runs CTA started
 * (min, median, max); end of a runs CTA incl. its hill slice (median, max);
 * finalize CTA duration (median, max); first finalize CTA start after the first
 * runs CTA started; coordination steps, runs grid, finalize CTAs per
 * walker, finalize grid; median durations of the finalize phases: loads and
 * walker record, CN and distance/angle/dihedral CVs, dU/dCV and energies,
 * coordination scatter, distance/angle/dihedral rows; median durations of the
 * runs CTAs' hill phases: wait for the staged data, hill-table evaluation,
 * lane reduction and store; second step: runs kernel, finalize kernel (events);
 * first coordination step's data landed after a runs CTA started, first step's
 * duration (medians)}. No reference counterpart.                               */
int glued_batch_phase_times(glued_batch* b, double* out);
/* Raw records of the last glued_batch_phase_times call: per runs CTA {SM id,
 * coordination steps, %globaltimer at entry, staging issued, coordination done,
 * hill data ready, hill evaluation done, exit, first step's data landed, first
 * step and its hill-CV evaluation done, first step done}, then per finalize CTA six
 * %globaltimer stamps. *n = number of values; min(cap, *n) are copied to out
 * (out may be NULL when cap is 0). No reference counterpart.                   */
int glued_batch_phase_stamps(glued_batch* b, unsigned long long* out, long long cap, long long* n);

#ifdef __cplusplus
}
#endif
#endif /* GLUED_B200_H */
