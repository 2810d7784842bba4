/* fastlbp_b200.h - C ABI of the B200 causal loopy-belief-propagation engine.
 *
 * This is the drop-in boundary underneath the libDAI-style C++ API
 * (include/ext/causal_bp.h). Every entry point uses plain pointers and sizes,
 * returns an int status (FLBP_OK == 0) and never exits the process; the
 * message of the last failure on the calling thread is available from
 * flbp_last_error(). Host arrays passed in are copied; the engine owns its
 * device buffers. One engine handle must be driven by one host thread at a
 * time; all of its GPU work goes to the stream given at creation (or to a
 * stream the engine creates).
 *
 * FastLBP has no C ABI of its own: each entry point below names the
 * reference member function (path:line within the FastLBP project) whose
 * job it takes over.
 */
#ifndef FASTLBP_B200_H
#define FASTLBP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FLBP_OK 0
#define FLBP_ERR_INVALID 1 /* bad argument or malformed graph */
#define FLBP_ERR_CUDA 2    /* CUDA runtime error */
#define FLBP_ERR_NOMEM 3   /* device or host allocation failed */
#define FLBP_ERR_STATE 4   /* call not valid in the engine's current state */
#define FLBP_ERR_LIMIT 5   /* graph exceeds an engine limit (e.g. 2^32-1 edge slots) */
#define FLBP_ERR_TIMEOUT 6 /* a device-side bounded wait gave up */

/* Factor types, as returned by CausalFactor::type() (csrc/ext/causal_factor.cpp:39-50). */
#define FLBP_SINGLETON 0
#define FLBP_AND 1
#define FLBP_OR 2

/* Stop reasons of the run entry points. */
#define FLBP_ALL_CONVERGED 0
#define FLBP_BIG_FRAC_CONVERGED 1
#define FLBP_DIVERGED 2 /* iteration or time limit reached */

/* Update schedules (the "updates" property, csrc/ext/causal_bp.cu:144-184) */
#define FLBP_UPDATES_PARALL 0
#define FLBP_UPDATES_SEQFIX 1
#define FLBP_UPDATES_TOPO 2

/* A causal factor graph in the reference's factor-major edge order: the
 * arrays CausalBP::construct() derives (csrc/ext/causal_bp.cu:310-407).
 * Factor I owns edge slots [factor_offsets[I], factor_offsets[I+1]) holding
 * the indices of vars(I) in ascending label order; factor_head[I] is the
 * absolute slot of its head variable. */
typedef struct flbp_graph_desc {
    int64_t n_vars;
    int64_t n_factors;
    int64_t n_slots;                    /* == factor_offsets[n_factors] */
    const int64_t *factor_offsets;      /* n_factors + 1   (row_ptr_vf)          */
    const int64_t *slot_var;            /* n_slots         (col_ind_vf)          */
    const int64_t *factor_head;         /* n_factors       (h_head)              */
    const int32_t *factor_type;         /* n_factors       FLBP_SINGLETON/AND/OR */
    const double *factor_p;             /* n_factors       prob()                */
    const double *factor_q;             /* n_factors       prob_default()        */
    const int32_t *factor_head_clamped; /* n_factors, may be NULL (none clamped) */
    const double *factor_mask0;         /* n_factors, may be NULL; head_mask[0], 0 or 1 */
    const double *factor_mask1;         /* n_factors, may be NULL; head_mask[1], 0 or 1 */
} flbp_graph_desc;

typedef struct flbp_engine_opts {
    int32_t precision; /* 32: FP32 log-odds messages (default); 64: FP64 */
    int32_t device;    /* CUDA device ordinal, -1 = current device */
    double damping;    /* f->v damping d in [0,1): log-odds mix (1-d)*new + d*old */
    void *stream;      /* cudaStream_t to use, NULL = engine-owned stream */
} flbp_engine_opts;

typedef struct flbp_run_info {
    int64_t sweeps;       /* sweeps performed by this call */
    int64_t total_sweeps; /* sweeps since init() (the reference's _iters) */
    double maxdiff;       /* last max |belief change| (NaN when not computed) */
    double frac;          /* the reference's yetToConvergeFraction */
    int32_t reason;       /* FLBP_ALL_CONVERGED / BIG_FRAC_CONVERGED / DIVERGED */
    int32_t status;       /* device status word (0 = ok) */
    int64_t launches;     /* engine kernels launched by this call */
} flbp_run_info;

typedef struct flbp_engine flbp_engine;

/* Thread-local text of the last error. */
const char *flbp_last_error(void);

/* Library version string. */
const char *flbp_version(void);

/* Build the device layout of a graph and allocate its message buffers.
 * Replaces CausalBP::construct() + putParallUpdateSeqToKernelFused()
 * (csrc/ext/causal_bp.cu:310-407, 724-817). */
int flbp_engine_create(const flbp_graph_desc *graph, const flbp_engine_opts *opts, flbp_engine **out);

/* Release every device and host resource of the engine. */
int flbp_engine_destroy(flbp_engine *eng);

/* Reset all messages to uniform, beliefs to 0 and the sweep count to 0.
 * Replaces CausalBP::init() (csrc/ext/causal_bp.cu:824-856). */
int flbp_init(flbp_engine *eng);

/* Tolerance-driven loop: sweep while sweeps < maxiter, max |belief change| >
 * tol and elapsed < maxtime seconds. Replaces CausalBP::run()
 * (csrc/ext/causal_bp.cu:858-910). As the reference's _iters, `sweeps`
 * counts every sweep since the engine was constructed (init() does not
 * reset it), and the first sweep's belief change is taken against the
 * beliefs the engine holds (0 in a new engine). */
int flbp_run_tol(flbp_engine *eng, double tol, int64_t maxiter, double maxtime, flbp_run_info *info);

/* The run state a new engine starts with: sweep count 0 and beliefs 0, so
 * that init() + flbp_run_tol gives what a newly constructed engine gives
 * (the reference resets both only on construction,
 * csrc/ext/causal_bp.cu:371). Messages are left to init(). */
int flbp_reset_counts(flbp_engine *eng);

/* Exactly `sweeps` sweeps, then one belief evaluation; low-pass beliefs equal
 * the beliefs and the returned fraction is 1. Replaces
 * CausalBP::run(tol, maxIters, histLength) (csrc/ext/causal_bp.cu:912-1004). */
int flbp_run_fixed(flbp_engine *eng, int64_t sweeps, flbp_run_info *info);

/* Convergence loop with the big-fraction rule and the low-pass belief
 * history mean. Replaces CausalBP::run(tol, minIters, maxIters, histLength)
 * (csrc/ext/causal_bp.cu:1006-1143). */
int flbp_run_lowpass(flbp_engine *eng, double tol, int64_t min_iters, int64_t max_iters, int64_t hist_length,
                     double maxtime, flbp_run_info *info);

/* `n` bare sweeps (f->v, per-variable totals, v->f) with no belief work.
 * Replaces calcNewMessageFusedAll() (csrc/ext/causal_bp.cu:409-444). */
int flbp_sweep(flbp_engine *eng, int64_t n);

/* Beliefs P(x=1) of all variables after the last run, in graph variable
 * order. Replaces transferBeliefToHost() / beliefV()
 * (csrc/ext/causal_bp.cu:521-554). */
int flbp_get_beliefs(flbp_engine *eng, double *out, int64_t n_vars);

/* Low-pass beliefs of the last run (newBelief(), include/ext/causal_bp.h:182-184). */
int flbp_get_lowpass(flbp_engine *eng, double *out, int64_t n_vars);

/* Beliefs evaluated now from the current messages (no run needed). */
int flbp_compute_beliefs(flbp_engine *eng, double *out, int64_t n_vars);

/* Current f->v messages as (P(x=0), P(x=1)) pairs in the reference's
 * variable-major slot order. Replaces transferMessagesToHost()
 * (csrc/ext/causal_bp.cu:1145-1161). */
int flbp_get_fv_messages(flbp_engine *eng, double *m0, double *m1, int64_t n_slots);

/* Current v->f messages in the reference's factor-major slot order (slots to
 * singleton factors and to factors whose outputs are constant report the
 * variable's message all the same). */
int flbp_get_vf_messages(flbp_engine *eng, double *m0, double *m1, int64_t n_slots);

/* Layout statistics: counts[0..17] = vars, factors, slots, active factors,
 * active slots, factors handled warp-wide, variables handled warp-wide,
 * bytes of device memory held, host->device bytes copied by create, engine
 * kernels launched so far, warp-wide factors too large for a tile, likewise
 * variables, tiles of warp-wide factors, tiles of warp-wide variables, and
 * the wall time (microseconds) of create's phases: host layout, device
 * allocation, host->device copies (with their host-side packing), and the
 * rest (device and stream set-up, kernel configuration, initial state),
 * then the tiles of the factor pass and the tiles of the variable pass.
 * Entries past n_counts are not written. */
int flbp_engine_stats(flbp_engine *eng, int64_t *counts, int64_t n_counts);

/* Per-pass timing mode (for measurement): while enabled, every sweep is
 * launched from a CUDA graph captured for the call that also records CUDA
 * events (event nodes) around the factor and the variable pass, so the
 * passes run back to back as in the normal graph-replayed sweeps. Enabling
 * resets the accumulators. */
int flbp_set_kernel_timing(flbp_engine *eng, int32_t enable);

/* Accumulated device time (ms) and launch counts of the factor pass [0] and
 * the variable pass [1] recorded in timing mode. */
int flbp_kernel_times(flbp_engine *eng, double *ms, int64_t *counts);

/* ---- kernel configuration of the PARALL sweep ----
 *
 * FastLBP launches every sweep kernel with a fixed kCudaThreadsNum = 128
 * threads per block, one thread per edge or variable
 * (include/utils/cuda_utils.h:23-27, csrc/kernel/causal_bp_parall.cu:400-467).
 * Here each of the two passes of a sweep has two forms with identical
 * results: 0 = staged (persistent blocks in which a producer warp bulk-copies
 * tiles of items into a shared-memory ring for 16 consumer warps) and direct
 * (every warp of a persistent grid loads its own items straight into
 * registers; 1 = up to 64 registers per thread, two 16-warp blocks per SM,
 * 2 = up to 40 registers, three blocks per SM). Which is faster depends on
 * the graph; new engines start with both passes staged. */
typedef struct flbp_tuning {
    int32_t factor_form; /* 0 staged, 1 or 2 direct */
    int32_t var_form;    /* 0 staged, 1 or 2 direct */
    int32_t factor_blocks; /* flbp_get_tuning: blocks launched per factor pass (ignored when set) */
    int32_t var_blocks;    /* flbp_get_tuning: blocks launched per variable pass (ignored when set) */
} flbp_tuning;

int flbp_set_tuning(flbp_engine *eng, const flbp_tuning *tuning);
int flbp_get_tuning(flbp_engine *eng, flbp_tuning *tuning);

/* Autotuner: times the forms of the two passes on this engine's own graph
 * and installs the fastest (coordinate descent: the factor pass's form
 * first, then the variable pass's). kind 0 times whole fixed-sweep runs
 * (init + `sweeps` sweeps + beliefs); kind 1 whole tolerance runs (tol,
 * maxiter = sweeps; batched engines: flbp_batch_run_tol, whose cost changes
 * as graphs stop, which is why whole runs are timed). Each candidate runs
 * once to capture its graphs, then `reps` timed runs; the median decides.
 * The choice is cached in the process by precision, damping, batching,
 * kind and a size class of the graph (log2 of variables and slots, share of
 * slots in warp-wide items), and later engines of the same class take it
 * without timing. The engine is left as flbp_init leaves it, with its sweep
 * count and previous beliefs as before the call. No counterpart in FastLBP
 * (it hard-codes kCudaThreadsNum = 128, include/utils/cuda_utils.h:23). */
int flbp_autotune(flbp_engine *eng, int32_t kind, int64_t sweeps, double tol, int32_t reps, flbp_tuning *chosen);

/* ------------------------------------------------------------------------
 * Allocation-free solve. No counterpart in FastLBP.
 *
 * For callers that may not allocate GPU memory when they solve: serving
 * loops whose policy forbids allocation after start-up (cudaMalloc
 * synchronises the device), and processes or plugin hosts whose GPU memory
 * belongs to another allocator. The caller
 * passes the graph and the belief output as device arrays it owns; the two
 * message arrays live in a fixed scratch array inside the library (2 x
 * FLBP_NOALLOC_MAX_SLOTS floats = 4 MiB, held by every GPU that loads the
 * library until the process exits). Nothing is allocated or freed.
 *
 * - Graphs with more than FLBP_NOALLOC_MAX_SLOTS edge slots are rejected
 *   with FLBP_ERR_LIMIT.
 * - The first call on a device looks up the scratch address on that device
 *   (cudaGetSymbolAddress, with the device current); make that first call
 *   before any stream capture.
 * - All calls share the one scratch array and it keeps the last call's
 *   messages; each call resets them to uniform first. Calls whose GPU work
 *   overlaps (different streams or host threads without ordering) race on
 *   the scratch and give wrong results: order them.
 * - Work is launched on `stream` (NULL: the legacy default stream); the
 *   call returns without waiting for it.
 * - The device arrays are trusted, not checked (that would need a device
 *   pass and a read-back): the graph must be well formed - factor_offsets
 *   non-decreasing from 0 to n_slots; factor_head[I] inside factor I's
 *   slots; var_offsets non-decreasing from 0 to n_slots; var_slots a
 *   permutation of 0..n_slots-1 grouped by variable; factor types 0-2 with
 *   singletons of one slot; p, q in [0,1]. A malformed graph makes the
 *   kernels read and write outside the arrays and the scratch.
 * ---------------------------------------------------------------------- */
#define FLBP_NOALLOC_MAX_SLOTS (1 << 19)

/* A graph in device memory, in the reference's orders (the arrays of
 * CausalBP::construct()), 32-bit. */
typedef struct flbp_device_graph {
    int32_t n_vars, n_factors, n_slots;
    const int32_t *factor_offsets;     /* n_factors + 1: factor-major slot offsets (row_ptr_vf) */
    const int32_t *slot_var;           /* n_slots: variable of each slot (col_ind_vf); not read, may be NULL */
    const int32_t *factor_head;        /* n_factors: absolute slot of each factor's head */
    const int32_t *factor_type;        /* n_factors: FLBP_SINGLETON / FLBP_AND / FLBP_OR */
    const uint8_t *factor_head_state;  /* n_factors or NULL: 0 free, 1 head clamped to 1, 2 to 0, 3 mask (0,0) */
    const float *factor_p;             /* n_factors: prob() */
    const float *factor_q;             /* n_factors: prob_default() */
    const int32_t *var_offsets;        /* n_vars + 1: variable-major offsets (row_ptr_fv) */
    const int32_t *var_slots;          /* n_slots: factor-major slot of each variable-major entry */
} flbp_device_graph;

/* `sweeps` synchronous sweeps from uniform messages with f->v damping
 * `damping`, then beliefs P(x=1) into beliefs_out (n_vars doubles, device).
 * FP32 log-odds messages, the same arithmetic as the engine. */
int flbp_run_fixed_device_noalloc(const flbp_device_graph *graph, int64_t sweeps, double damping,
                                  double *beliefs_out, void *stream);

/* Device duration in milliseconds of the engine's GPU work recorded by the
 * last run call (CUDA events on the engine stream). */
int flbp_last_run_ms(flbp_engine *eng, double *ms);

/* ------------------------------------------------------------------------
 * Graph model (host). The libDAI-style CausalFactorGraph of the C++ API,
 * exposed for callers without C++ (Python ctypes, other FFIs).
 * ---------------------------------------------------------------------- */

typedef struct flbp_fg flbp_fg;

/* Read a .causal_fg file. Replaces CausalFactorGraph::ReadFromFile()
 * (csrc/ext/causal_fg.cpp:118-127, 129-279). */
int flbp_fg_read_file(const char *path, flbp_fg **out);

/* Parse .causal_fg text held in memory. */
int flbp_fg_read_string(const char *text, flbp_fg **out);

/* Build from parallel factor arrays (bodies as label CSR; body_off has n+1
 * entries). Replaces CausalFactorGraph(const std::vector<CausalFactor>&)
 * (csrc/ext/causal_fg.cpp:50-68). */
int flbp_fg_from_factors(int64_t n, const int32_t *type, const int64_t *head, const int64_t *body_off,
                         const int64_t *body, const double *p, const double *q, flbp_fg **out);

int flbp_fg_destroy(flbp_fg *fg);

/* Clamp variable index i to x (0/1). Replaces CausalFactorGraph::clamp()
 * (csrc/ext/causal_fg.cpp:17-26). Topology is left as it was, as in the
 * reference; flbp_fg_rebuild() then gives fl_wrapper's rebuilt graph. */
int flbp_fg_clamp(flbp_fg *fg, int64_t i, int64_t x);

/* New graph from this graph's factors (CausalFactorGraph(fg.factors()),
 * examples/fl_wrapper.cu:45). */
int flbp_fg_rebuild(const flbp_fg *fg, flbp_fg **out);

/* Sizes: counts[0..3] = vars, factors, edges (sum of neighbour lists),
 * slots (sum of |vars(factor)|). */
int flbp_fg_sizes(const flbp_fg *fg, int64_t *counts);

int flbp_fg_var_labels(const flbp_fg *fg, int64_t *labels, int64_t n);

/* Per-factor fields; vars_off has n_factors+1 entries, vars has n_slots. */
int flbp_fg_factors(const flbp_fg *fg, int32_t *type, int64_t *head, double *p, double *q, int32_t *clamped,
                    double *mask0, double *mask1, int64_t *vars_off, int64_t *vars);

/* Neighbour lists (node, iter, dual) of variables (which = 0) or factors
 * (which = 1), in CSR form. */
int flbp_fg_neighbors(const flbp_fg *fg, int32_t which, int64_t *off, int64_t *node, int64_t *iter, int64_t *dual);

/* The factor-major arrays of CausalBP::construct() for this graph's factors
 * (topology rebuilt from vars(), as fl_wrapper does): offsets (F+1),
 * slot_var, head, plus the per-variable CSR of the variable-major order
 * (row_ptr_fv, V+1) and its factor column (col_ind_fv). */
int flbp_fg_construct(const flbp_fg *fg, int64_t *factor_offsets, int64_t *slot_var, int64_t *factor_head,
                      int64_t *row_ptr_fv, int64_t *col_ind_fv);

/* Engine straight from a graph-model handle (what CausalBP's constructor does). */
int flbp_engine_create_from_fg(const flbp_fg *fg, const flbp_engine_opts *opts, flbp_engine **out);

/* ---- batched solves (no counterpart in the reference: it solves one graph
 * per CausalBP object, csrc/ext/causal_bp.cu:858-910) ----
 *
 * One engine over n_graphs independent graphs (their disjoint union, graphs
 * in order): every sweep is one pass over all of them, and each graph stops
 * by itself under the reference's tolerance rule, after which its messages
 * and beliefs stay frozen. A graph's results are those of solving it alone
 * with flbp_run_tol from init(). flbp_get_beliefs returns the beliefs of all
 * graphs, graph g's variables at [var_off[g], var_off[g+1]). */
int flbp_batch_create(const flbp_graph_desc *graphs, int64_t n_graphs, const flbp_engine_opts *opts,
                      flbp_engine **out);

/* Number of graphs and their variable ranges (var_off: n_graphs + 1 entries,
 * may be NULL). */
int flbp_batch_info(flbp_engine *eng, int64_t *n_graphs, int64_t *var_off);

/* Tolerance run of every graph from the current messages (call flbp_init
 * first for a fresh solve): graph g stops after the first sweep in which no
 * belief moved by more than tol, or after maxiter sweeps; the call returns
 * when all graphs have stopped or maxtime seconds have passed. Per graph:
 * sweeps[g] (NULL allowed) and reasons[g] (FLBP_ALL_CONVERGED or
 * FLBP_DIVERGED; NULL allowed). */
int flbp_batch_run_tol(flbp_engine *eng, double tol, int64_t maxiter, double maxtime, int64_t *sweeps,
                       int32_t *reasons, flbp_run_info *info);

/* ---- evidence sets on one graph (no counterpart in the reference: its
 * alarm-ranking loop clamps, rebuilds the graph and builds a new CausalBP
 * for every label set, examples/bingo_wrapper.cu:25-77, fl_wrapper.cu:29-45) ----
 *
 * One engine over n_sets evidence sets of one graph: the graph's layout is
 * stored once, each set has its own messages, priors and beliefs. Set k
 * clamps the variables set_vars[set_off[k] .. set_off[k+1]) (graph variable
 * order) to set_vals[...] (0 or 1) with the effect of flbp_clamp_vars on an
 * engine of its own (the clamp rewrite of csrc/ext/causal_factor.cpp:63-100
 * followed by a rebuild). flbp_init resets every set (uniform messages,
 * the clamped variables' v->f messages +-inf, beliefs 0 as in a new
 * engine); flbp_sets_run_tol then runs the reference's tolerance rule with
 * each set stopping by itself (sweeps[k], reasons[k] as in
 * flbp_batch_run_tol; NULL allowed), so that set k has the beliefs and
 * sweep count of its own engine solved alone.
 * flbp_get_beliefs returns n_sets * n_vars values, set k at
 * [k n_vars, (k+1) n_vars). Runs use the direct form of both passes with
 * the sets as the second grid dimension; calls of a single graph's run
 * state (flbp_run_*, flbp_sweep, gradients, clamps, export, schedules)
 * return FLBP_ERR_STATE. At most 65535 sets. */
int flbp_sets_create(const flbp_graph_desc *graph, int64_t n_sets, const int64_t *set_off, const int64_t *set_vars,
                     const int32_t *set_vals, const flbp_engine_opts *opts, flbp_engine **out);
int flbp_sets_run_tol(flbp_engine *eng, double tol, int64_t maxiter, double maxtime, int64_t *sweeps,
                      int32_t *reasons, flbp_run_info *info);
/* Number of sets (0 for other engines) and variables per set; either pointer may be NULL. */
int flbp_sets_info(flbp_engine *eng, int64_t *n_sets, int64_t *n_vars);

/* ---- gradients through unrolled sweeps (no counterpart in the reference) ----
 *
 * flbp_adjoint_forward: init() and `sweeps` synchronous sweeps (engines
 * without damping), keeping the v->f messages every `every` sweeps; writes
 * the beliefs after the last sweep (n = number of variables; may be NULL).
 * flbp_adjoint_backward: given dL/dbelief for every variable, the gradient
 * of L with respect to every factor's p and q (reference factor order; NULL
 * allowed, and a NULL grad_q also skips accumulating dL/dq), by reversing
 * the sweeps of the last forward run: each segment
 * between checkpoints is recomputed, then the adjoint kernels run backwards
 * through it. Singleton priors and AND/OR factors reduced to their head get
 * their p gradient through the folded constant logit(p). */
int flbp_adjoint_forward(flbp_engine *eng, int64_t sweeps, int64_t every, double *beliefs, int64_t n);
int flbp_adjoint_backward(flbp_engine *eng, const double *grad_beliefs, double *grad_p, double *grad_q);

/* flbp_adjoint_backward on device buffers of the engine's device, in the
 * same orders (grad_p / grad_q may be NULL). The caller's writes to
 * grad_beliefs must be complete before the call; the gradients are complete
 * when it returns. */
int flbp_adjoint_backward_device(flbp_engine *eng, const double *grad_beliefs, double *grad_p, double *grad_q);

/* flbp_get_beliefs into a device buffer of the engine's device. */
int flbp_get_beliefs_device(flbp_engine *eng, double *out, int64_t n_vars);

/* Where new engines build their device layout (process-wide; no counterpart
 * in FastLBP, whose construct() builds its edge records on the host,
 * csrc/ext/causal_bp.cu:310-407, 724-817): 0 (default) on the GPU for graphs
 * of at least 2^18 edge slots and on the host below that, 1 always on the
 * host, 2 always on the GPU. Both builds give the same layout bit for bit.
 * A GPU-built engine keeps the caller's graph arrays in device memory and
 * builds the complete host-side layout only when a call needs it (message
 * export, gradients, clamps, schedules, new probabilities). Batched engines
 * always build on the host. */
int flbp_set_layout_builder(int32_t mode);

/* Digest (64-bit FNV-1a) of an engine's device layout as its kernels read
 * it: every layout buffer copied back, and the layout's counts; equal
 * digests mean equal layouts. *built_on_device (may be NULL): 1 when the
 * engine's layout was built on the GPU. */
int flbp_engine_layout_digest(flbp_engine *eng, uint64_t *digest, int32_t *built_on_device);

/* A digest (64-bit FNV-1a) of the device layout the engine would build for
 * `graph` (no counterpart in the reference; needs no GPU), built on the host
 * with `threads` threads (0: all). For batches, factor_graph / var_graph give
 * every factor's and variable's graph (n_graphs > 0), else NULL and 0. The
 * layout does not depend on the thread count; tests use this to check it. */
int flbp_layout_digest(const flbp_graph_desc *graph, const uint32_t *factor_graph, const uint32_t *var_graph,
                       uint32_t n_graphs, int32_t threads, uint64_t *digest);

/* ---- incremental evidence (the alarm-ranking loop) ----
 *
 * Clamps variables (graph variable order) to 0 or 1 on an existing engine,
 * with the effect of CausalFactorGraph::clamp on every neighbouring factor
 * followed by a rebuild and a new engine (csrc/ext/causal_factor.cpp:63-100,
 * csrc/ext/causal_fg.cpp:17-26; fl_wrapper.cu:29-45 and bingo_wrapper.cu
 * rebuild after every label), without the rebuild: the variable gets an
 * exact-zero count in its prior and no factor's message reaches it any
 * more. An input at +-inf leaves a noisy-AND/OR product unchanged or zeroes
 * it, which is exactly the reference's removal of the variable from a body
 * or its "killed" factor (p := q, empty body). Takes effect from the next
 * init()/run; like a new engine, the engine then counts its sweeps against
 * maxiter from zero and its tolerance rule starts from beliefs 0 (the
 * reference resets both only when an engine is constructed,
 * csrc/ext/causal_bp.cu:371). Clamping a variable again to the same value changes nothing;
 * to the other value is rejected (FLBP_ERR_INVALID). Messages exported
 * afterwards (flbp_get_fv_messages) keep the unclamped graph's slots. */
int flbp_clamp_vars(flbp_engine *eng, int64_t n, const int64_t *vars, const int32_t *values);

/* New p and q for every factor (reference order) of an existing engine, e.g.
 * after a learning step: constants folded into priors follow. The graph's
 * structure (which factors are singletons, clamped or reduced) stays. */
int flbp_set_factor_probs(flbp_engine *eng, const double *p, const double *q);
/* The same with p and q in the engine's device memory (F doubles each,
 * complete when the call is made: the engine's stream does not wait for
 * another stream). The range check runs on the device (one 8-byte read
 * back); the update itself stays on the device: (p, q) in the internal
 * and big-tile orders, the folded singletons' prior constants (the sum of
 * sign (log p - log1p(-p)) over each variable's prior entries) and their
 * derivatives for the adjoint. The host copies are refreshed only when a
 * later call needs them (a sequential schedule). */
int flbp_set_factor_probs_device(flbp_engine *eng, const double *p, const double *q);

/* ---- Sequential schedules (updates=SEQFIX / TOPO) ----------------------
 * An update sequence lists every edge once, as its factor-major slot
 * (factor_offsets[I] + position in the factor). */

/* The update sequence of a schedule. FLBP_UPDATES_SEQFIX: the slots of
 * factor_order[0], then of factor_order[1], ... (a permutation of the
 * factors; buildFixedUpdateSeq, csrc/ext/causal_bp.cu:186-201, shuffles it
 * with the thread's std::mt19937). FLBP_UPDATES_TOPO: edges ranked by a
 * breadth-first order over variables and factors (buildTopoUpdateSeq,
 * csrc/ext/causal_bp.cu:203-304); factor_order is ignored. seq_out holds
 * n_slots entries. */
int flbp_update_seq(const flbp_graph_desc *graph, int32_t kind, const int32_t *factor_order, int64_t *seq_out);

/* 0..n-1 shuffled by std::shuffle with std::mt19937(seed): the SEQFIX factor
 * order of the first CausalBP a thread constructs after seeding rnd_gen. */
int flbp_shuffled_factors(int64_t n, uint32_t seed, int32_t *order);

/* The conflict-free batches the engine runs a sequence in
 * (putUpdateSeqToKernelFused, csrc/ext/causal_bp.cu:583-722): batch of every
 * slot (n_slots entries, may be NULL) and their number. Host only. */
int flbp_seq_batches(const flbp_graph_desc *graph, const int64_t *seq, int64_t n, int64_t *slot_batch,
                     int64_t *n_batches);

/* Run this engine's sweeps in the batches of `seq` (n == n_slots), one batch
 * after the other: the batch's v->f messages from the current variable
 * totals, then its f->v messages, each folded into its variable's total at
 * once (calcNewMessageFused, csrc/ext/causal_bp.cu:446-476, and
 * csrc/kernel/causal_bp_seq.cu). seq == NULL returns to PARALL. Resets the
 * messages to the init() state. Not available on batched engines, after
 * flbp_clamp_vars, or together with the adjoint and flbp_set_factor_probs
 * (FLBP_ERR_STATE). */
int flbp_set_update_seq(flbp_engine *eng, const int64_t *seq, int64_t n);

/* How sequential sweeps are launched: 0 chooses (the default: one cluster per
 * sweep when batches are small, else two launches per batch), 1 two kernel
 * launches per batch over the whole GPU, 2 the whole sweep as one launch on
 * one thread-block cluster, 3 as 1 with programmatic dependent launch.
 * Results are the same. */
int flbp_set_seq_kernel(flbp_engine *eng, int32_t kind);

/* Whether the engine runs an installed sequence (1) or PARALL (0), and its
 * number of batches per sweep (1 for PARALL). Either pointer may be NULL. */
int flbp_update_info(flbp_engine *eng, int32_t *sequential, int64_t *n_batches);

#ifdef __cplusplus
}
#endif

#endif /* FASTLBP_B200_H */
