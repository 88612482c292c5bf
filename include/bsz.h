/*
 * bsz.h -- C ABI of the B200 bitstream executor (libbsz.so).
 *
 * Plain C types only (pointers, sizes, int64).  No exceptions cross this
 * boundary: every function returns a status (0 = OK, nonzero = error; NULL
 * for constructors) and bsz_last_error() returns the message of the last
 * failure on the calling thread.  A context owns one CUDA stream and all
 * device buffers it allocates; it is not thread-safe.
 *
 * Streams are little-endian arrays of uint64 words: bit i of a stream is bit
 * (i % 64) of word (i / 64).  A stream of bitlength N has ceil(N/64) words.
 * Beyond its stored words a stream carries a "tail" bit (0 or 1): the value
 * of every higher bit, which is how the reference's normative Python
 * semantics represent negative integers (infinitely many ones).
 *
 * Reference interfaces replaced (paths relative to the reference project):
 *  - the bsim_cuda process contract  simulator/csim/src/main.cu:209-331
 *    (argv + JSON on stdout)          -> bsz_run_case_json(), and the
 *                                        bsim_cuda executable built on it
 *  - Interpreter<Backend>::run        simulator/csim/src/interpreter.inl:234-364
 *                                     -> bsz_compile / bsz_run_* / bsz_execute
 *  - the CudaBackend data plane       simulator/csim/src/cuda_backend.cuh:16-229
 *    (op_not/and/or/xor/add/shl/shr,   -> bsz_op_* entry points on device
 *     op_popcount, op_is_nonzero)          pointers
 */
#ifndef BSZ_H_
#define BSZ_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bsz_ctx bsz_ctx;
typedef struct bsz_program bsz_program;
typedef struct bsz_run bsz_run;

/* Execution forms. */
#define BSZ_MODE_PLAIN 0   /* one kernel per DSL operation */
#define BSZ_MODE_FUSED 1   /* whole straight-line segments as one generated kernel */
#define BSZ_MODE_AUTO 2    /* device interpreter (one launch per segment) for streams of at
                              most 8192 words; generated kernels for longer ones when cached
                              or worth compiling; else one kernel per operation */
#define BSZ_MODE_VM 3      /* every segment on the device interpreter */

typedef struct bsz_stats {
  int64_t op_count;          /* dynamic DSL op count (same counting as the reference) */
  int64_t n_kernel_launches; /* kernels launched by this execution */
  int64_t n_mallocs;         /* cudaMalloc calls made by the context so far */
  int64_t n_segments;        /* device segments executed */
  int64_t n_syncs;           /* host<->device synchronisations */
  int64_t peak_bytes;        /* peak device bytes held in stream buffers */
  int64_t max_live;          /* peak number of live stream buffers */
  double kernel_ms;          /* CUDA-event time of the execution */
  double compile_ms;         /* time spent generating/compiling fused kernels */
  int64_t n_fused_launches;  /* generated segment kernels launched */
  int64_t n_fused_fallbacks; /* segment parts re-run per-op because speculation was unproven */
  int64_t n_vm_launches;     /* segments run by the device interpreter */
  int64_t walk_replayed;     /* 1: a straight-line program's statement walk was restored from
                                the program's walk cache (same bit length, mode and bindings as
                                an earlier run); the device work runs in full either way */
} bsz_stats;

/* Schedule of the generated segment kernels (fused form).  The autotuner and
 * the learned cost model choose among these; zero-initialised fields of a
 * default schedule are {4, 64, 0, 4, 1, 0}. */
typedef struct bsz_schedule {
  int32_t warps;        /* warps per CTA (1..16) */
  int32_t range_steps;  /* minimum 32-word steps owned by one warp (words per tile / 32) */
  int32_t ctas_per_sm;  /* resident CTAs per SM, 0 = as many as occupancy allows, -1 = no
                           persistent cap: one minimum-length range per warp */
  int32_t min_blocks;   /* launch-bounds minimum blocks per SM (caps registers) */
  int32_t prefetch;     /* 1: load the next 32-word step before computing this one */
  int32_t cut_adds;     /* carry scheme: 0, additions inside the fused kernels (speculative
                           carry state, exact re-run if unproven); 1, the same with every
                           addition's result materialized (one kernel per addition level);
                           2, every addition of two streams run by the plain single-pass
                           carry-scan kernel (decoupled look-back) on materialized operands */
  int32_t layout;       /* 0: each warp walks a word range, lane = word (cross-word state by
                           ballots and shuffles); 1: each thread walks its own word range
                           (cross-word state in registers, 256-bit per-thread accesses);
                           2: as 1, with every input and output moved by TMA boxes of
                           chunk_words words x 32 threads through shared memory */
  int32_t chunk_words;  /* layout 1: 4 or 8 words per thread per register chunk (one or two
                           256-bit accesses per stream); layout 2: 4 or 8 words per thread
                           per box; any other value reads as 4 */
  int32_t stages;       /* layout 2: 2 or 3 shared-memory stages of input boxes */
  int32_t unroll;       /* layout 2: 1 = the word pairs of a chunk are unrolled */
  int32_t shift_mul;    /* layouts 1-2: 1 = shifts as integer multiply-adds (the multiply
                           pipe) instead of funnel shifts (the logic pipe) */
} bsz_schedule;

/* ---- library ---------------------------------------------------------- */
const char* bsz_version(void);
const char* bsz_last_error(void);

/* ---- context ---------------------------------------------------------- */
/* Creates a context on CUDA device `device` (must be sm_100). */
bsz_ctx* bsz_create(int device);
void bsz_destroy(bsz_ctx* ctx);
/* The context's cudaStream_t, as void*. */
void* bsz_stream(bsz_ctx* ctx);
int bsz_sync(bsz_ctx* ctx);
/* Per-kernel timing with CUDA events on the context's stream: enable != 0
 * starts (and resets) it.  bsz_profile_report() synchronizes and returns
 * JSON {"kernel name": {"launches": n, "ms": total}}, owned by the library. */
int bsz_profile(bsz_ctx* ctx, int enable);
const char* bsz_profile_report(bsz_ctx* ctx);

/* ---- programs (replaces bs::parse, simulator/csim/src/parser.cpp:451-457) */
/* Parses and validates DSL source.  NULL on ParseError / ThreeAddrError. */
bsz_program* bsz_compile(bsz_ctx* ctx, const char* source, size_t len);
void bsz_program_free(bsz_program* prog);
/* Static op count for the given params (ast_liveness.cpp:629-727). */
int64_t bsz_static_ops(bsz_program* prog, const char* const* param_names,
                       const int64_t* param_values, int n_params);

/* ---- one execution (replaces Interpreter<CudaBackend>::run) -------------- */
bsz_run* bsz_run_create(bsz_program* prog, int64_t bitlength, int mode);
void bsz_run_free(bsz_run* run);
int bsz_set_param(bsz_run* run, const char* name, int64_t value);
/* Sets the fused-kernel schedule for this run (before bsz_execute). */
int bsz_run_set_schedule(bsz_run* run, const bsz_schedule* schedule);
/* Binds an input stream.  index < 0: scalar input; index >= 0: element of an
 * input array.  `words` holds n_words words on the host (on_device = 0, the
 * copy is made on the context's stream) or on the device (on_device = 1, the
 * buffer is copied so the caller keeps ownership; on_device = 2, the device
 * buffer is borrowed without a copy and must stay valid and unchanged until
 * bsz_run_free).  Words beyond n_words are zero (or all ones when tail = 1);
 * words past ceil(bitlength/64) are ignored.  Names the program does not
 * declare as inputs are ignored, as the reference executors ignore them. */
int bsz_bind_input(bsz_run* run, const char* name, int64_t index, const uint64_t* words,
                   uint64_t n_words, int tail, int on_device);
/* Binds a broadcast array (bsdata "_broadcast_pack"): element i is all-ones
 * (-1) when ones[i] != 0, else zero. */
int bsz_bind_broadcast(bsz_run* run, const char* name, const uint8_t* ones, int64_t count);
/* Runs the program.  stats may be NULL. */
int bsz_execute(bsz_run* run, bsz_stats* stats);
/* Asynchronous form of bsz_execute: walks the program and enqueues its device
   work on the context's stream, then returns without waiting (no host
   read-back), so the host can prepare the next run while the device works.
   bsz_run_wait waits, checks the fused kernels' speculation (re-running
   unproven parts exactly), reads the popcounts and fills `stats` (may be
   NULL).  Reading a result of a launched run waits implicitly.  A run's
   inputs must stay unchanged until it has finished. */
int bsz_execute_async(bsz_run* run);
int bsz_run_wait(bsz_run* run, bsz_stats* stats);
/* Results.  For a stream output: copies ceil(bitlength/64) words (bits at and
 * above the bitlength cleared, as the reference masks outputs) into host
 * memory.  index < 0 for scalar outputs.  Returns nonzero if absent. */
int bsz_get_stream(bsz_run* run, const char* name, int64_t index, uint64_t* host,
                   uint64_t n_words);
/* Device pointer of a stream output (valid until bsz_run_free). */
int bsz_get_stream_device(bsz_run* run, const char* name, int64_t index,
                          const uint64_t** dptr);
int bsz_get_int(bsz_run* run, const char* name, int64_t* value);
/* Indices present in an array output; returns the count (<= cap written),
 * or -1 if the array does not exist. */
int64_t bsz_array_indices(bsz_run* run, const char* name, int64_t* indices, int64_t cap);

/* ---- batches: many independent instances in one launch ------------------
 * Several straight-line programs (no if/while on streams, no input/output
 * arrays, no right shift of a temporary) run over many instances of
 * different stream lengths by ONE persistent kernel that holds every
 * program's DAG and pulls (instance, word range) items from a work queue.
 * bsz_batch_create traces and compiles once and captures the launch in a
 * CUDA graph; bsz_batch_launch replays it (asynchronous); bsz_batch_finish
 * waits and reads every instance's popcount results.  No reference
 * counterpart: the reference runs one process per case
 * (benchmark/base.py:228-254). */
typedef struct bsz_instance {
  int32_t program;                 /* index into the programs array */
  int64_t bitlength;               /* this instance's stream length in bits */
  const uint64_t* const* inputs;   /* device pointers, one per declared scalar input */
  uint64_t* const* outputs;        /* device pointers, one per declared output stream (NULL: skip) */
} bsz_instance;
typedef struct bsz_batch bsz_batch;
bsz_batch* bsz_batch_create(bsz_ctx* ctx, bsz_program* const* programs, int n_programs,
                            const bsz_instance* instances, int64_t n_instances,
                            const bsz_schedule* schedule);
int bsz_batch_launch(bsz_batch* batch);
int bsz_batch_finish(bsz_batch* batch, bsz_stats* stats);
/* Output ints of one instance (declaration order); returns how many. */
int bsz_batch_ints(bsz_batch* batch, int64_t instance, int64_t* values, int capacity);
int64_t bsz_batch_items(bsz_batch* batch);
void bsz_batch_free(bsz_batch* batch);

/* ---- learned schedule cost model ------------------------------------------
 * A small FP32 MLP (in_dim -> hidden x layers (ReLU) -> 1) trained with Adam
 * on MSE by hand-written CUDA kernels on the context's stream.  x is n rows
 * of in_dim floats (row-major, host), y / out n floats (host).  No reference
 * counterpart. */
/* DAG features of a straight-line program for the cost model (traced and
 * simplified as the fused form sees it): writes up to `capacity` floats,
 * returns the number of features (BSZ_NUM_FEATURES) or -1 on error. */
#define BSZ_NUM_FEATURES 15
int bsz_program_features(bsz_ctx* ctx, bsz_program* prog, float* out, int capacity);
typedef struct bsz_mlp bsz_mlp;
bsz_mlp* bsz_mlp_create(bsz_ctx* ctx, int in_dim, int hidden, int layers, uint64_t seed);
int64_t bsz_mlp_num_params(bsz_mlp* mlp);
/* One Adam step; *loss = the batch loss before the step. */
int bsz_mlp_train_step(bsz_mlp* mlp, const float* x, const float* y, int n, float lr, float* loss);
int bsz_mlp_predict(bsz_mlp* mlp, const float* x, int n, float* out);
/* Loss and its gradient w.r.t. the flat parameters (no update). */
int bsz_mlp_gradients(bsz_mlp* mlp, const float* x, const float* y, int n, float* grad, float* loss);
/* Flat parameters W1 b1 W2 b2 ... Wout bout (each W row-major [fan_in, fan_out]);
 * get != 0 copies them out, get == 0 loads them (and resets Adam state). */
int bsz_mlp_params(bsz_mlp* mlp, float* params, int get);
/* Decoupled (AdamW) weight decay applied by bsz_mlp_train_step (default 0). */
int bsz_mlp_set_weight_decay(bsz_mlp* mlp, float weight_decay);
void bsz_mlp_free(bsz_mlp* mlp);

/* ---- whole-case driver (replaces run_case<64>, main.cu:23-207) ----------
 * Runs `source` on every case of a .bsdata file (or, if bsdata_path is NULL,
 * on the JSON input document `json_input`, the stdin form of main.cu) and
 * returns the bsim_cuda JSON text (one object, or an array for multi-case
 * files).  flags: bit 0 = --warmup, bits 1-2 = execution mode (BSZ_MODE_*).  The returned string
 * is owned by the library and valid until the next call on this thread. */
const char* bsz_run_case_json(bsz_ctx* ctx, const char* source, const char* bsdata_path,
                              const char* json_input, int flags);

/* ---- per-op data plane on device pointers (CudaBackend op_*) -----------
 * dst/a/b are device pointers to n_words words; `bitlength` is the logical
 * length (bits at and above it are cleared by ~, + and <<): 1 .. 64*n_words,
 * or 0 for the full storage width; anything else is an error.  dst may be
 * a or b exactly (in place); partially overlapping buffers are not allowed.
 * All calls are asynchronous on the context's stream except popcount /
 * is_nonzero, which return their result to the host. */
int bsz_op_not(bsz_ctx* ctx, uint64_t* dst, const uint64_t* a, uint64_t n_words,
               int64_t bitlength);
int bsz_op_and(bsz_ctx* ctx, uint64_t* dst, const uint64_t* a, const uint64_t* b,
               uint64_t n_words);
int bsz_op_or(bsz_ctx* ctx, uint64_t* dst, const uint64_t* a, const uint64_t* b,
              uint64_t n_words);
int bsz_op_xor(bsz_ctx* ctx, uint64_t* dst, const uint64_t* a, const uint64_t* b,
               uint64_t n_words);
int bsz_op_andnot(bsz_ctx* ctx, uint64_t* dst, const uint64_t* a, const uint64_t* b,
                  uint64_t n_words);
int bsz_op_add(bsz_ctx* ctx, uint64_t* dst, const uint64_t* a, const uint64_t* b,
               uint64_t n_words, int64_t bitlength);
int bsz_op_shl(bsz_ctx* ctx, uint64_t* dst, const uint64_t* a, uint64_t k, uint64_t n_words,
               int64_t bitlength);
int bsz_op_shr(bsz_ctx* ctx, uint64_t* dst, const uint64_t* a, uint64_t k, uint64_t n_words,
               int tail);
int bsz_op_popcount(bsz_ctx* ctx, const uint64_t* a, uint64_t n_words, uint64_t* result);
int bsz_op_is_nonzero(bsz_ctx* ctx, const uint64_t* a, uint64_t n_words, int* result);

/* Byte -> basis-bit transposition on the device (replaces
 * payload_to_basis_bits / payload_to_basis_bits_fast,
 * benchmark/apps/regex/src/run.py:164-187): bit j of basis stream i = bit i
 * of bytes[j].  `bytes` (n_bytes) and the eight `basis[i]` (ceil(n_bytes/64)
 * words each) are device pointers; bits at and above n_bytes are zero.
 * Asynchronous on the context's stream. */
int bsz_s2p(bsz_ctx* ctx, const uint8_t* bytes, int64_t n_bytes, uint64_t* const* basis);

/* Stream addition that allocates no device memory (no counterpart in the
 * reference).  For callers that cannot allocate GPU memory when they call:
 * a serving process whose pool already holds almost all of HBM, a host
 * application that passes its own buffers through FFI and owns every
 * allocation, or a loop that cannot pay for the device-wide synchronisation
 * of cudaMalloc/cudaFree.  Same result as bsz_op_add (dst = a + b with bits
 * at and above `bitlength` cleared; the same bitlength and in-place rules);
 * no context is needed.  The look-back scratch is a fixed file-scope device
 * array of about 1 MiB, so n_words is limited to 2^26 (streams of up to
 * 2^32 bits); longer streams are rejected with an error.  The CUDA runtime
 * loads the library's device code on a device lazily, and that load commits
 * the array, which the device then keeps until the process exits: the first
 * call on each device therefore allocates that 1 MiB once.  Callers that
 * must never allocate later make one set-up call per device at start-up,
 * while allocation is still allowed and before any stream capture; a call
 * with n_words = 0 does only that set-up (pointers unused).  Every call
 * reuses the same array, so calls that overlap on the GPU (different
 * streams, or different host threads) race; serialize them.  Runs on
 * `stream` (a cudaStream_t, NULL for the default stream) and returns when
 * the addition has finished. */
int bsz_add_noalloc(uint64_t* dst, const uint64_t* a, const uint64_t* b, uint64_t n_words,
                    int64_t bitlength, void* stream);

/* Test hook for the add kernel's bounded look-back waits (no counterpart in
 * the reference; tests only).  Until reset with silent_tile = -1, tile
 * `silent_tile` of every add never publishes its carry status and a wait
 * gives up after `spin_limit` spins (<= 0: the normal limit), so the tile
 * after it reports a look-back timeout: bsz_op_add's context and
 * bsz_add_noalloc then return an error naming it.  Not thread-safe. */
void bsz_debug_add_lookback_hook(int64_t silent_tile, int spin_limit);

#ifdef __cplusplus
}
#endif

#endif /* BSZ_H_ */
