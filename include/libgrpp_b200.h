/*
 * Batched C-ABI of the B200 GRPP integral engine.
 *
 * libgrpp (aoleynichenko/libgrpp) evaluates one shell pair x one potential
 * centre per call (libgrpp/libgrpp.h:123-231) and leaves parallelism to the
 * caller (test_libgrpp_c/eval_integrals.c:78-83). This header adds batched
 * entry points with no counterpart in libgrpp: a whole list of
 * (shell A, shell B, centre C) tasks is described once in flat arrays
 * (plain pointers and sizes, host memory) and evaluated on the GPU in one
 * call. The single-task libgrpp_* functions of libgrpp.h are implemented on
 * top of these with a batch of one.
 *
 * Task semantics are those of libgrpp_full_grpp_integrals
 * (libgrpp/full_grpp_integrals.c:27-104): for task t the four output blocks
 * hold arep, so_x, so_y, so_z of <A| U_GRPP(C) |B>, row-major
 * cart_size(A) x cart_size(B), stored consecutively in task order:
 * block t starts at sum_{s<t} cart_size(A_s) * cart_size(B_s).
 */
#ifndef LIBGRPP_B200_BATCH_H
#define LIBGRPP_B200_BATCH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    /* ---- shells: basis shells and outercore shells share one table ----
     * coefficients are the raw contraction coefficients a caller passes to
     * libgrpp_new_shell (no normalisation folded in). */
    int n_shells;
    const int *shell_L;          /* [n_shells] */
    const int *shell_nprim;      /* [n_shells] */
    const int *shell_prim_off;   /* [n_shells] offset into prim_coef / prim_alpha */
    const double *prim_coef;
    const double *prim_alpha;
    const double *shell_origin;  /* [3*n_shells]; ignored for outercore shells */
    const int *shell_cart_off;   /* [n_shells] offset (in components) into cart_list */
    const int *cart_list;        /* 3 ints (x,y,z powers) per Cartesian component */

    /* ---- potentials sum_k c_k r^(n_k-2) exp(-zeta_k r^2) ---- */
    int n_pots;
    const int *pot_L;
    const int *pot_J;            /* 2j for outercore potentials, 0 otherwise */
    const int *pot_nprim;
    const int *pot_prim_off;
    const int *pot_powers;       /* n_k in {0,1,2} */
    const double *pot_coef;
    const double *pot_alpha;

    /* ---- GRPP operators (one per element) ---- */
    int n_grpps;
    const int *grpp_UL;          /* [n_grpps] potential index of U_L, -1 if none */
    const int *grpp_arep_off;    /* into grpp_pot_list */
    const int *grpp_n_arep;
    const int *grpp_so_off;      /* into grpp_pot_list */
    const int *grpp_n_so;
    const int *grpp_oc_off;      /* into grpp_oc_pot / grpp_oc_shell */
    const int *grpp_n_oc;
    const int *grpp_pot_list;
    const int *grpp_oc_pot;
    const int *grpp_oc_shell;

    /* ---- potential centres ---- */
    int n_centres;
    const double *centre_origin; /* [3*n_centres] */
    const int *centre_grpp;      /* [n_centres] */

    /* ---- tasks ---- */
    int64_t n_tasks;
    const int *task_a;           /* bra shell */
    const int *task_b;           /* ket shell */
    const int *task_c;           /* centre */
} libgrpp_b200_batch_t;

/* status codes */
enum {
    LIBGRPP_B200_OK = 0,
    LIBGRPP_B200_ERR_INVALID = 1,    /* input outside the supported limits */
    LIBGRPP_B200_ERR_CUDA = 2,       /* a CUDA runtime call failed */
    LIBGRPP_B200_ERR_TIMEOUT = 3,    /* a bounded device-side wait gave up */
    LIBGRPP_B200_ERR_NOT_INIT = 4    /* libgrpp_init() was not called */
};

/* radial quadrature modes */
enum {
    LIBGRPP_B200_RADIAL_PLAIN = 0,   /* level-by-level nested Log3 doubling */
    LIBGRPP_B200_RADIAL_LEARNED = 1  /* walk scheduled by the learned level model (same results) */
};

/* last error of the calling thread: code and message */
int libgrpp_b200_last_error(void);
const char *libgrpp_b200_last_error_message(void);

/* total number of doubles of one output array for this batch */
int64_t libgrpp_b200_batch_output_size(const libgrpp_b200_batch_t *batch);

/* Full GRPP integrals for every task (host in, host out). Returns a status code. */
int libgrpp_b200_full_grpp_batch(const libgrpp_b200_batch_t *batch, int radial_mode, double *arep,
                                 double *so_x, double *so_y, double *so_z);

/* Page-locked host memory for input and output arrays of the calls above: device<->host
 * copies to and from it run at full link speed and need no staging. Returns NULL on
 * failure (message in libgrpp_b200_last_error_message). Free with libgrpp_b200_host_free.
 * Not part of libgrpp's interface. */
void *libgrpp_b200_host_alloc(size_t bytes);
void libgrpp_b200_host_free(void *p);

/* Select the CUDA device used by the calling thread (this library keeps its own
 * CUDA runtime state; default device 0). Returns a status code. */
int libgrpp_b200_set_device(int device);

/* Measured FP64 FMA throughput of the current device in TFLOP/s (8 independent FMA chains
 * per thread, all SMs busy): the denominator of this engine's roofline. */
int libgrpp_b200_fp64_peak(double *tflops);

/* A batch prepared once on the device: inputs uploaded and work lists built, device
 * buffers owned by the plan. execute() runs the kernels only (outputs stay on the
 * device until outputs() copies them to host arrays). Not thread-safe per plan. */
typedef struct libgrpp_b200_plan libgrpp_b200_plan_t;

libgrpp_b200_plan_t *libgrpp_b200_plan_create(const libgrpp_b200_batch_t *batch, int radial_mode);

/* plan_create with a fixed block size of the assembly kernel for every task (128, 256 or
 * 512 threads); 0 uses the autotuner's per-class table, or the default rule where the table
 * has no entry for a class. */
libgrpp_b200_plan_t *libgrpp_b200_plan_create_ex(const libgrpp_b200_batch_t *batch, int radial_mode,
                                                 int assembly_threads);

/* Per-class autotuner of the assembly kernel (no counterpart in libgrpp). A class is
 * (la, lb, largest semilocal L of the centre's GRPP, spin-orbit terms or not). Every class
 * of `batch` runs as a launch of its own with 128, 256 and 512 threads per block, timed
 * with CUDA events; the fastest size per class is kept for the later batches and plans of
 * this device. Writes up to `cap` rows of 6 doubles: class key ((la*16+lb)*16+L)*2+so,
 * tasks, milliseconds at 128, 256, 512 threads, chosen size. Returns the number of classes
 * or a negative status code. */
int libgrpp_b200_autotune_assembly(const libgrpp_b200_batch_t *batch, int radial_mode, double *rows, int cap);

/* Forget the autotuner's table of the current device (the default rule applies again). */
void libgrpp_b200_autotune_reset(void);
int libgrpp_b200_plan_execute(libgrpp_b200_plan_t *plan);
int libgrpp_b200_plan_outputs(libgrpp_b200_plan_t *plan, double *arep, double *so_x, double *so_y, double *so_z);
/* ms[5] = kernel time of the last execute(): total, type 1, radial (screening + grid walk),
 * assembly, screening alone (CUDA events on the engine stream); counts[5] = tasks, radial tasks, type 1 work items, radial entries, bytes uploaded */
int libgrpp_b200_plan_stats(const libgrpp_b200_plan_t *plan, double *ms, int64_t *counts);
/* operation counters of the radial kernel in the last execute() (n <= 16 slots): screening and
 * grid-walk SM cycles, tasks, integrand points, Bessel evaluations, primitive Gaussians, potential
 * terms, r^N powers, entry x point accumulations, screening estimates / iterations / envelopes, levels */
int libgrpp_b200_plan_counters(const libgrpp_b200_plan_t *plan, uint64_t *counters, int n);
void libgrpp_b200_plan_destroy(libgrpp_b200_plan_t *plan);
/* on != 0: later executes also count the type 1 kernel's operations (slots 13-14 of
 * libgrpp_b200_plan_counters: primitive triples, FP64 operations) in a slower build of
 * that kernel; the radial counters are always kept. */
int libgrpp_b200_plan_set_counting(libgrpp_b200_plan_t *plan, int on);

/* Density-contracted GRPP gradient (no counterpart in libgrpp, whose driver forms one
 * gradient matrix per atom coordinate, test_libgrpp_c/main.c:529-620):
 *   g[m][atom][k] += sum over tasks (A, B, C) sum_ij D[bf_off[A]+i][bf_off[B]+j] d V^m_ij / d R_atom,k
 * for the four matrices m = arep, so_x, so_y, so_z of libgrpp_full_grpp_integrals and
 * every atom: the same quantity as libgrpp_full_grpp_integrals_gradient contracted
 * with D for each atom of A, B and C (the only atoms that can contribute,
 * grpp_integrals_gradient.c:311-321). shell_atom[n_shells] and centre_atom[n_centres]
 * map shells and centres to atoms, atom_xyz[3*n_atoms] are their positions (a shell's
 * origin and its atom's position coincide), bf_off[n_shells] is each shell's first
 * basis function, D is n_bf x n_bf row-major, g is [4][n_atoms][3] and is accumulated
 * into. Shells of the tasks must have L <= 9. Returns a status code. */
int libgrpp_b200_grpp_gradient_contract(const libgrpp_b200_batch_t *batch, int radial_mode, const int *shell_atom,
                                        const int *centre_atom, const double *atom_xyz, int n_atoms, const int *bf_off,
                                        int n_bf, const double *D, double *g);

/* One-electron integrals over the batch's shell pairs (task_a, task_b; task_c is not read
 * and the batch may have no centres), blocks laid out as in libgrpp_b200_full_grpp_batch.
 * Per pair the values of libgrpp_overlap_integrals (overlap.c:39-62),
 * libgrpp_kinetic_energy_integrals (kinetic.c:34-57) and libgrpp_momentum_integrals
 * (momentum.c:34-68; out0..out2 = x, y, z), computed on the GPU. */
enum {
    LIBGRPP_B200_ONEE_OVERLAP = 0,
    LIBGRPP_B200_ONEE_KINETIC = 1,
    LIBGRPP_B200_ONEE_MOMENTUM = 2
};
int libgrpp_b200_onee_batch(const libgrpp_b200_batch_t *batch, int kind, double *out0, double *out1, double *out2);

/* Nuclear attraction over every task (A, B, C): the nucleus of charge centre_charge[C] at
 * centre C, libgrpp_nuclear_attraction_integrals per task (nuclear_attraction.c:31-119).
 * nuclear_model is a LIBGRPP_NUCLEAR_MODEL_* value; centre_params[3*C..] holds the model's
 * parameters (ball, Gaussian: R_rms; Fermi: c, a; Fermi bubble: c, a, k; ignored for point
 * charges). Point charges run through the type 1 McMurchie-Davidson kernel with a zero
 * exponent, the other models through the numeric type 1 kernel. centre_grpp is not read. */
int libgrpp_b200_nuclear_attraction_batch(const libgrpp_b200_batch_t *batch, int nuclear_model,
                                          const double *centre_charge, const double *centre_params, double *out);

/* <A| U_L |B> of the centre GRPP's local part by numeric radial quadrature instead of
 * McMurchie-Davidson: libgrpp's evaluate_type1_integral_primitive_gaussians scheme
 * (type1_integrals.c:109-270, radial_type1_integral.c:73-325) per primitive pair; the
 * independent evaluation of the same integrals libgrpp_type1_integrals gives. L_A + L_B <= 12. */
int libgrpp_b200_type1_numeric_batch(const libgrpp_b200_batch_t *batch, double *arep);

/* The same gradient for a symmetric density (checked: |D_ij - D_ji| <= 1e-14 max|D|, else
 * LIBGRPP_B200_ERR_INVALID). A task (B, A, C) then contributes to tr(D V_arep) what (A, B, C)
 * does, and every spin-orbit contraction tr(D V_so) vanishes (the SO matrices are
 * antisymmetric): the ordered tasks are folded onto A <= B (each shell-pair block and its
 * derivatives evaluated once, weight 2 where both orders are listed), no spin-orbit
 * potential is evaluated, and g[1..3][..] (so_x, so_y, so_z), whose exact value is zero,
 * receive no contribution. */
int libgrpp_b200_grpp_gradient_contract_symmetric(const libgrpp_b200_batch_t *batch, int radial_mode,
                                                  const int *shell_atom, const int *centre_atom, const double *atom_xyz,
                                                  int n_atoms, const int *bf_off, int n_bf, const double *D, double *g);

/* Learned grid-level model (no counterpart in libgrpp).
 *
 * libgrpp's type 2 radial quadrature (radial_type2_integral.c:242-318) doubles a
 * nested Log3 grid level by level until every entry of a task has converged; the
 * deepest level a task needs (0..8, i.e. 31..8191 points) is known only after the
 * walk. The level model is an MLP (12 features -> 64 -> 64 -> 64 -> 9 levels, BF16
 * weights, FP32 accumulation) that predicts it. LIBGRPP_B200_RADIAL_LEARNED uses the
 * prediction to schedule the walk (tasks taken from a work queue, deepest predicted
 * level first); every task is still walked until libgrpp's own stop rule ends it, so
 * the results equal those of LIBGRPP_B200_RADIAL_PLAIN bit for bit.
 *
 * Parameter vector (FP32, LIBGRPP_B200_LEVEL_MODEL_PARAMS floats):
 *   mean[12] std[12] W1[64][12] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[9][64] b4[9]
 * Features of a task (radial work item): la, lb, max projector L, number of semilocal
 * potentials, log(1+|CA|), log(1+|CB|), log of the min and max exponent of shell A, of
 * shell B and of the potential terms; normalised as (f - mean) / std. */
#define LIBGRPP_B200_LEVEL_MODEL_PARAMS 9761
#define LIBGRPP_B200_LEVEL_FEATURES 12

/* Install the model used by LIBGRPP_B200_RADIAL_LEARNED on the current device. */
int libgrpp_b200_set_level_model(const float *params);

/* Training data: run the batch with the plain walk; for each task that has semilocal
 * potentials (in task order; *n_items of them, at most n_tasks) write its features
 * (12 floats) and the level libgrpp's stop rule ended its walk at (-1 when every
 * entry was settled by screening or analytically). */
int libgrpp_b200_level_samples(const libgrpp_b200_batch_t *batch, float *features, int8_t *levels,
                               int64_t *n_items);

/* Mean cross-entropy and its gradient w.r.t. the (BF16-rounded) weights of the model
 * on n samples (levels 0..8), computed by the training kernels; grad has
 * LIBGRPP_B200_LEVEL_MODEL_PARAMS floats (the normalisation slots are 0). */
int libgrpp_b200_mlp_grad(const float *params, const float *features, const int8_t *levels, int n, float *grad,
                          float *loss);

/* Adam training on the GPU (forward/backward/update kernels of this library): params
 * holds the initial weights and the normalisation on entry and the trained FP32
 * weights on return; epoch_loss[e] receives the mean cross-entropy of epoch e. */
int libgrpp_b200_mlp_train(const float *features, const int8_t *levels, int64_t n, int epochs, int batch, float lr,
                           uint32_t seed, float *params, float *epoch_loss);

/* Predicted levels of n feature rows (the BF16 inference path the walk uses). */
int libgrpp_b200_mlp_predict(const float *params, const float *features, int64_t n, int8_t *levels);

/* Learned-mode statistics of the last execute(): time of the prediction and ordering
 * kernels (ms) and the number of tasks whose walk went beyond the predicted level + 1. */
int libgrpp_b200_plan_learned_stats(const libgrpp_b200_plan_t *plan, double *ms_predict, int64_t *fallbacks);

/* Allocation-free type 2 integrals (no counterpart in libgrpp).
 *
 * For callers that must not trigger device allocations: processes whose device
 * memory is owned by a pool or framework allocator, and services that must keep a
 * fixed device footprint. For every task of the batch, arep receives the sum over
 * the centre GRPP's averaged (AREP) semilocal potentials of the type 2 integrals
 * (libgrpp_type2_integrals summed as libgrpp_full_grpp_integrals does); U_L,
 * spin-orbit and outercore parts are not evaluated. Host arrays in and out, blocks
 * laid out as in libgrpp_b200_full_grpp_batch.
 *
 * The call allocates no device memory: all device data live in static device
 * arrays loaded with the library, including one 32 MiB scratch array that holds
 * the call's inputs, working state and outputs. Batches needing more are
 * rejected with LIBGRPP_B200_ERR_INVALID (split them); so are malformed batches,
 * checked on the host before any CUDA call. The first call on a device sets that
 * device up (tables copied, scratch address taken); make it before any stream
 * capture. The call is synchronous (cudaMemcpy, legacy default stream) and
 * returns when the results are on the host. All calls share the scratch array:
 * host calls are serialised, and calls overlapping on the GPU would race. */
int libgrpp_b200_type2_batch_noalloc(const libgrpp_b200_batch_t *batch, double *arep);

#ifdef __cplusplus
}
#endif

#endif /* LIBGRPP_B200_BATCH_H */
