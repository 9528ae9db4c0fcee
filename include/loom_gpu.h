/*
 * loom_gpu.h — C ABI of the B200 (sm_100a) implementation of loom's
 * Poseidon2-backend prove phase (github.com/consensys/loom).
 *
 * The Go prover binds these functions through a cgo shim package; Python
 * binds them through ctypes (loom_b200/_lib.py).  Signatures use plain pointers and
 * sizes only.  Every function returns an int status (LG_OK = 0) and never
 * aborts; lg_last_error() describes the last failure on a context.
 *
 * Field data: KoalaBear (p = 2^31 - 2^24 + 1) elements are 32-bit
 * Montgomery words (R = 2^32), the in-memory layout of gnark-crypto's
 * koalabear.Element, so Go slices are passed as they are.  An E6 element is
 * 6 such words [B0.A0, B0.A1, B1.A0, B1.A1, B2.A0, B2.A1] (ext.E6).  A
 * digest is 8 words (hash.Digest).
 *
 * Data buffers flagged `on_device` are device pointers on the context's GPU;
 * otherwise host pointers.  Small parameter arrays (challenges such as
 * alpha and z, row counts, widths, and the arrays of column pointers
 * themselves) are always host memory.  Input pointers are only read during
 * the call; device witness columns given to lg_prove are used in place and
 * must not change until it returns.
 *
 * Program descriptor (lg_prove): little-endian u32 words —
 *   magic 0x3150474C, n_rounds, n_modules, n_columns, n_nodes, n_steps
 *   module  : log2(N), str name, n_rel, rel_root[n_rel]
 *   column  : str name, module, field (0 base | 1 ext),
 *             kind (0 witness | 1 prover-step output | 2 Lagrange verifier
 *             column | 3 setup column, precommitted by lg_setup), param
 *             (int32 row for kind 2; negative -(i+1) counts from the last row)
 *   node    : op (0 column | 1 round coin | 2 constant | 3 add | 4 sub |
 *             5 mul | 6 exposed average | 7 exposed value), a, b — column:
 *             a = column, b = int32 shift; coin: a = round; constant: a =
 *             canonical value; add/sub/mul: a, b = earlier nodes; exposed
 *             average: a = exposed value index, the constant value / N of
 *             the exposing step's module (expr/ast.go:223-227); exposed
 *             value: a = exposed value index, the value as a constant
 *             (times L_0 it is expr.Exposed, board/product.go:109)
 *   step    : type 0 grand product (board/step.go:301-327): 0, round,
 *             module, numerator node, denominator node, output column
 *             type 1 lookup multiplicities of width-1 tables
 *             (board/board.go:235-249): 1, round, n_src, n_tgt,
 *             source nodes, target nodes, output column per target
 *             type 2 cyclic logup column (board/logup.go:80-180): 2, round,
 *             module, output column, n_terms (<= 4 on the GPU), then
 *             (denominator node, numerator node) per term; its total is
 *             exposed in the proof and bound after the round's commitment
 *             type 3 running ratio (board/product.go:72-198): 3, round,
 *             module, numerator node, denominator node, output column; its
 *             end is exposed.  Exposed values are numbered in step order
 *             over types 2 and 3.
 *             type 4 lookup multiplicities of tuples with optional selectors
 *             (internal/poly/lookup_multiplicity.go:37-100): 4, round, width
 *             (<= 8), n_src, n_tgt, flags (bit 0 source selectors, bit 1
 *             target selectors), source selector nodes, target selector
 *             nodes (when flagged), source nodes (width per table), target
 *             nodes (width per table), output column per target
 *   round   : n_staged, staged column indices (board.Compile's order,
 *             including the sweep of unstaged columns into the last round)
 *   str     : byte length, then the bytes packed 4 per word
 * This is the part of a compiled board.Program (board/program.go:21-89)
 * that the prove phase reads.  Witness columns (kind 0) are passed to
 * lg_prove in descriptor order, N words each, Lagrange form.
 *
 * Proof bytes: the canonical encoding defined by this project — 4-byte
 * big-endian words, field elements in canonical (non-Montgomery) form, in
 * the field order of proof.Proof / fri.OpeningProof / fri.Proof; lists are
 * a count followed by the items (see loom_b200/proof.py for a decoder).
 */
#ifndef LOOM_GPU_H
#define LOOM_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  LG_OK = 0,
  LG_ERR_INVALID = 1,     /* malformed arguments or program */
  LG_ERR_CUDA = 2,        /* CUDA runtime failure */
  LG_ERR_OOM = 3,         /* device allocation failed */
  LG_ERR_UNSUPPORTED = 4, /* shape or hash backend this build does not handle */
  LG_ERR_BUFFER = 5       /* output buffer too small; size written back */
};

typedef struct lg_ctx lg_ctx;
/* A committed batch kept on the device: every group's LDE, coefficients and
 * the Merkle tree (fri.Committed, internal/fri/pcs.go:131-168). */
typedef struct lg_committed lg_committed;
/* One prove of one program in progress, driven phase by phase by a caller
 * that keeps the Fiat-Shamir transcript (the Go prover's runtime,
 * prover/prover.go:142-719). */
typedef struct lg_session lg_session;

/* Creates a context (one CUDA stream, twiddle caches, memory pool) on
 * `device`.  `hbm_budget` caps the device bytes the context may hold at once
 * (0: no cap); an allocation past it fails with LG_ERR_OOM.  Replaces nothing
 * in the reference: the Go prover has no device state; the cgo shim creates
 * one context per GPU.  Release every handle made on a context before
 * destroying it. */
int lg_ctx_create(int device, size_t hbm_budget, lg_ctx** out);
void lg_ctx_destroy(lg_ctx* ctx);
/* Launch partitioning of every phase: batched (1, the default) launches each
 * kernel once over all groups / modules of a size class; plain (0) launches
 * it once per group / module, like a per-column prover.  Both produce the
 * same proof bytes. */
int lg_ctx_set_batched(lg_ctx* ctx, int batched);
/* Thread mapping of Poseidon2 leaf hashing and of the Merkle levels and
 * injection chains outside the one-block tree top: 1 = one thread per
 * permutation chain, 6 = six lanes of a warp per permutation, 0 = choose from
 * the number of independent chains per launch (default).  Results do not
 * depend on it. */
int lg_ctx_set_leaf_mapping(lg_ctx* ctx, int lanes_per_permutation);
/* Launch-shape choices (no counterpart in the reference: the autotuner in
 * loom_b200/autotune.py sets them from measurements).  Proof bytes never
 * depend on them.  Names and ranges:
 *   "p2_leaf_min_per_sm"  one thread per leaf / injection chain when a launch
 *                         has at least this many per SM (else six lanes)
 *   "p2_node_min_per_sm"  the same for one-permutation Merkle levels
 *   "p2_inject_min_per_sm" the same for the injection chains
 *   "merkle_tail"         levels narrower than this (power of two, 2..1024)
 *                         run in one block
 *   "merkle_subtree"      above that, one launch builds the levels over
 *                         this many nodes per block (power of two, 2..1024;
 *                         0: a launch per level)
 *   "inject_block", "leaf_block"  threads per block (power of two, 32..1024)
 *   "lde_split"           1: the LDE of 2^4..2^14 rows as an inverse launch
 *                         plus one block per (lane, coset); 0: one block per
 *                         lane for all of it
 *   "lde_fwd_threads"     threads per coset block (256, 512 or 1024)
 *   "fri_tail_leaves"     the FRI rounds whose layer tree has at most this many
 *                         leaves run in one block, back to back (power of two,
 *                         2..65536; 0: a launch per step of every round)
 *   "quotient_jit"        1: the constraint bytecode of each module's quotient
 *                         and of each grand product's ratio is compiled to a
 *                         kernel of its own at run time (NVRTC, cached per
 *                         program); 0: the bytecode interpreter
 *   "upload_split"        1: lg_prove with a host witness copies the columns
 *                         the first round commits first and the others on a
 *                         second stream while that round runs; 0: every
 *                         column before the prove starts
 * Unknown names or values out of range return LG_ERR_INVALID. */
int lg_ctx_set_tuning(lg_ctx* ctx, const char* name, int64_t value);
int lg_ctx_get_tuning(lg_ctx* ctx, const char* name, int64_t* value);
/* Free and total device memory of the context's GPU. */
int lg_mem_info(lg_ctx* ctx, uint64_t* free_bytes, uint64_t* total_bytes);
/* Device bytes a new allocation on `device` can get now — free memory plus
 * the unused reserve of the device's default memory pool, which every context
 * allocates from — and the total.  Needs no context and waits for no stream,
 * so a serving loop calls it at admission time while other proves run. */
int lg_device_mem_info(int device, uint64_t* available_bytes, uint64_t* total_bytes);
/* Device bytes the context holds now (buffers, caches, arena chunks) and
 * their high-water mark; reset_peak != 0 restarts the mark from now.  A
 * serving loop reads the mark around a prove to learn that prove's peak. */
int lg_ctx_mem_usage(lg_ctx* ctx, uint64_t* held_bytes, uint64_t* peak_bytes, int reset_peak);
/* NUL-terminated description of the last failure on `ctx` (never NULL). */
const char* lg_last_error(lg_ctx* ctx);

/* Whole prove phase for the Poseidon2 backend: replaces prover.Prove
 * (prover/prover.go:655-719) called with fri.Poseidon2HashBackend()
 * (internal/fri/hash_backend.go:21-40) and WithNumFriQueries(num_queries)
 * (prover/prover.go:74-80), no public inputs; setup columns come from
 * lg_setup.
 * `hash_backend` must be "poseidon2" (or "" = default); "sha256" and
 * "blake3" return LG_ERR_UNSUPPORTED.  The proof is written straight into
 * `proof` (capacity *proof_len; its length comes back in *proof_len).  On
 * LG_ERR_BUFFER it is kept in the context instead and lg_last_proof()
 * copies it out. */
int lg_prove(lg_ctx* ctx, const char* hash_backend, const uint32_t* program, size_t program_words,
             const uint32_t* const* witness, int witness_on_device, uint32_t num_queries, uint8_t* proof,
             size_t* proof_len);
int lg_last_proof(lg_ctx* ctx, uint8_t* proof, size_t* proof_len);
/* verifier.Verify (verifier/verifier.go:487-533) of proof bytes in the
 * canonical encoding against the program: transcript replay, buses, the AIR
 * relation at zeta and the FRI fold chains on the host; every Merkle opening
 * (committed batches with their injected groups, the levels tree, the FRI
 * layers) and the DEEP bridge of every query on the GPU.  `setup_root` (8
 * Montgomery words) is the verification key of a program with setup columns,
 * NULL otherwise; `buses` (may be NULL) lists product and logup buses as
 * "P:end,end;L:total,total,..." (board.Program's ProductBus and LogupBus).
 * Returns LG_OK when the proof is accepted; LG_ERR_INVALID with the reason in
 * lg_last_error() ("proof rejected: ...") when it is not. */
int lg_verify(lg_ctx* ctx, const uint32_t* program, size_t program_words, const uint8_t* proof, size_t proof_len,
              uint32_t num_queries, const uint32_t* setup_root, const char* buses);
/* setup.Setup (setup/setup.go:68-124) for a program with setup columns
 * (column kind 3: circuit constants such as selectors and permutations):
 * commits them, base field only, passed in descriptor order, into the setup
 * tree and keeps tree, LDE and columns on the context with the program (the
 * proving key); writes the root (the verification key, Montgomery words).
 * lg_prove of that program then takes only the witness columns (kind 0),
 * binds the root after the module sizes and leaves it out of the proof's
 * commitments.  The context keeps the setups of its eight most recently
 * proven programs; a program that dropped out needs lg_setup again. */
int lg_setup(lg_ctx* ctx, const uint32_t* program, size_t program_words, const uint32_t* const* setup_cols,
             int on_device, uint32_t root[8]);

/* ---- Phase-level entry points: the prover's phases with the transcript
 * kept by the caller.  Challenges go in by their transcript names; every
 * phase checks that the challenges it needs were given.  lg_prove runs the
 * same phases with the library's own transcript, so both routes give the
 * same proof bytes. */

/* PCS.Commit of one batch (internal/fri/pcs.go:145-168 ->
 * internal/fri/commitment.go:259-386): RS-encode every polynomial at rate 4,
 * hash adjacent row pairs into leaves with Poseidon2LeafHasher.HashLeafPairs
 * (internal/fri/hash.go:63-120) and build the mixed-height tree
 * (internal/merkle/tree.go:117-327), groups sorted by size, the largest the
 * leaf level.  Group g has rows[g] Lagrange rows, n_base[g] base columns then
 * n_ext[g] ext columns (ext.E6 rows, 6 words each) in `cols`, group by group.
 * Writes the root, and in *out a handle that keeps LDE, coefficients and tree
 * on the device for lg_committed_eval and lg_open_batches (PCS.Open,
 * internal/fri/open.go:98-105) until lg_release. */
int lg_commit(lg_ctx* ctx, uint32_t n_groups, const uint64_t* rows, const uint32_t* n_base, const uint32_t* n_ext,
              const uint32_t* const* cols, int on_device, lg_committed** out, uint32_t root[8]);
/* The root alone of the same commitment (nothing kept: no opening can
 * follow). */
int lg_commit_root(lg_ctx* ctx, uint32_t n_groups, const uint64_t* rows, const uint32_t* n_base,
                   const uint32_t* n_ext, const uint32_t* const* cols, int on_device, uint32_t root[8]);
/* Values of a committed batch's polynomials at zeta * w_N^s for each shift s
 * (w_N of the group's own size): computeClaimedValues
 * (internal/fri/values.go:46-110) for one batch.  out (E6, 6 words each):
 * group by group in declaration order, base polynomials then extension
 * polynomials, each at every shift. */
int lg_committed_eval(lg_ctx* ctx, const lg_committed* batch, const uint32_t zeta[6], uint32_t n_shifts,
                      const int32_t* shifts, uint32_t* out);
/* Openings of committed batches at FRI query positions s < 2^24
 * (openCommittedAt, internal/fri/open.go:290-378): per position the batch
 * count, then per batch the row pair of its largest group, that tree's
 * Merkle path with its injected leaves, and the other groups' row pairs —
 * in the canonical proof encoding.  LG_ERR_BUFFER writes the size needed. */
int lg_open_batches(lg_ctx* ctx, uint32_t n_batches, const lg_committed* const* batches, const uint32_t* positions,
                    uint32_t n_positions, uint8_t* out, size_t* out_len);

/* Starts a prove of `program` (descriptor as for lg_prove) over `witness`
 * (descriptor order; device witness columns are used in place and must stay
 * unchanged until lg_release of the session) with num_queries FRI queries:
 * newProverRuntime (prover/prover.go:142-275) without its transcript.  The
 * caller binds "poseidon2", the module sizes in layout order and, for a
 * program with setup columns, the setup root (lg_session_setup_root) to the
 * first challenge, as the reference does. */
int lg_session_begin(lg_ctx* ctx, const char* hash_backend, const uint32_t* program, size_t program_words,
                     const uint32_t* const* witness, int witness_on_device, uint32_t num_queries, lg_session** out);
/* The precommitted setup root of the session's program (*has_root = 0 when it
 * has no setup columns). */
int lg_session_setup_root(lg_session* s, uint32_t root[8], int* has_root);
/* A challenge the caller's transcript computed (fiatshamir ComputeChallenge,
 * internal/fiat-shamir/transcript.go:221-315), as its 8-word digest:
 * "challenge@loom_<r>", "__zeta", "alpha_DEEP", "fri_level_<l>_gamma",
 * "fri_fold_<j>". */
int lg_session_challenge(lg_session* s, const char* name, const uint32_t digest[8]);
/* Round r: ExecuteSteps and commitTraceRound (prover/prover.go:291-411) —
 * the round's generated columns, then its batch commitment (*committed = 1
 * and the root, which the caller binds to challenge@loom_<r>), then the
 * round's exposed values (6 words each, step order; capacity *n_exposed, the
 * count written back), which the caller binds after the root.  Needs the
 * challenges of rounds < r. */
int lg_commit_round(lg_session* s, uint32_t round, uint32_t root[8], int* committed, uint32_t* exposed,
                    uint32_t* n_exposed);
/* ComputeAIRQuotients (prover/prover.go:461-561 ->
 * poly.ComputeQuotientMixed, internal/poly/compute_quotient.go:223-424) and
 * the commitment of the quotient chunks; the caller binds the root to
 * __zeta.  Needs every round's challenge. */
int lg_quotient(lg_session* s, uint32_t root[8], int* committed);
/* computeClaimedValues (internal/fri/values.go:46-110) at zeta, written in
 * the order bindClaimedValuesByPolynomialOrder binds them to alpha_DEEP
 * (internal/fri/open.go:223-285): 6 words each; capacity *n_values, the
 * count written back. */
int lg_claimed_values(lg_session* s, uint32_t* values, size_t* n_values);
/* computeDeepQuotientCodewordsByPolynomial (internal/fri/deep.go:71-266) with
 * alpha_DEEP. */
int lg_deep(lg_session* s);
/* fri.Prove's levels tree over the DEEP codewords (internal/fri/fri.go:
 * 294-317,352-365): its root (the caller binds it to fri_level_1_gamma when
 * there are several levels, and to fri_fold_<first_round>), the level count
 * and the first round with a layer. */
int lg_fri_commit_levels(lg_session* s, uint32_t root[8], uint32_t* n_levels, uint32_t* first_round);
/* FRI round j (proveExt, internal/fri/fri.go:606-736): folds layer j with
 * challenge fri_fold_<j> (foldLayerExt, fri.go:1177-1198), adds the levels
 * that enter at j + 1 (their gammas must be set) and commits layer j + 1:
 * *committed = 1 with its root, which the caller binds to fri_fold_<j+1>;
 * 0 after the last round. */
int lg_fri_fold_round(lg_session* s, uint32_t round, uint32_t root[8], int* committed);
/* The FRI final polynomial after the last round (E6 values, 6 words each;
 * capacity *n_values, the count written back); the caller binds it to
 * fri_query_0 and derives the query positions. */
int lg_fri_final(lg_session* s, uint32_t* values, size_t* n_values);
/* The query openings at the caller's positions (openQueryExt,
 * internal/fri/fri.go:1251-1272; openCommittedAt, internal/fri/open.go:
 * 290-378) and the whole proof in the canonical encoding, as lg_prove writes
 * it (on LG_ERR_BUFFER lg_last_proof copies it out). */
int lg_open(lg_session* s, const uint32_t* positions, uint32_t n_positions, uint8_t* proof, size_t* proof_len);
/* A handle to the session's committed batch `index` (layout order: the setup
 * tree first when there is one, then the rounds' trees, then the AIR tree),
 * for lg_committed_eval and lg_open_batches; it keeps the batch's device
 * buffers after the session is released. */
int lg_session_committed(lg_session* s, uint32_t index, lg_committed** out);
/* Frees a handle (lg_committed or lg_session); NULL is ignored. */
void lg_release(void* handle);

/* reedsolomon.Encoder.Encode (internal/reedsolomon/rs.go:52-70) on
 * `n_cols` base columns of n_rows rows stored one after another in `in`;
 * writes 4 * n_rows bit-reversed evaluations per column to `out`. */
int lg_rs_encode(lg_ctx* ctx, const uint32_t* in, uint64_t n_rows, uint32_t n_cols, uint32_t* out, int on_device);

/* poseidon2.Permutation (width 24) applied in place to n_states states of
 * 24 words (the permutation behind internal/hash/poseidon2.go:165-449). */
int lg_poseidon2_permute(lg_ctx* ctx, uint32_t* states, uint64_t n_states, int on_device);

/* Merkle root over n_leaves digests with level injections
 * (merkle.NewWithInjections + Build, internal/merkle/tree.go:117-296):
 * n_inj injections of widths inj_widths[k] (non-increasing), their leaves
 * concatenated in `inj`.  A schedule validateInjections rejects
 * (internal/merkle/tree.go:140-160: a width that is not a power of two,
 * exceeds n_leaves or grows) returns LG_ERR_INVALID. */
int lg_merkle_root(lg_ctx* ctx, const uint32_t* leaves, uint64_t n_leaves, uint32_t n_inj,
                   const uint64_t* inj_widths, const uint32_t* inj, int on_device, uint32_t root[8]);

/* One FRI fold of n E6 evaluations in bit-reversed order
 * (foldLayerExt, internal/fri/fri.go:1177-1198); writes n/2 E6 values. */
int lg_fri_fold(lg_ctx* ctx, const uint32_t* layer, uint64_t n, const uint32_t alpha[6], uint32_t* out,
                int on_device);

/* DEEP quotient at one point over base columns in LDE form: for each row r
 * (x = w^bitrev(r) on the subgroup of order `rows`),
 * out[r] = sum_i alpha^i (values[i] - P_i(x)) / (z - x), where `lde` holds
 * n_cols columns of `rows` bit-reversed evaluations one after another and
 * values[i] = P_i(z) (E6; with on_device, all of lde, values and out are
 * device pointers).  The single-point form of
 * accumulateDeepQuotientByPolynomialOnTrace (internal/fri/deep.go:205-266),
 * evaluated on the LDE rows.  Writes `rows` E6 values. */
int lg_deep_quotient(lg_ctx* ctx, const uint32_t* lde, uint32_t n_cols, uint64_t rows, const uint32_t alpha[6],
                     const uint32_t z[6], const uint32_t* values, uint32_t* out, int on_device);

/* Grand product of a prover step: out[0] = 1, out[i] = prod_{k<i} num[k]/den[k]
 * over n E6 rows (6 words each, ext.E6 layout) — the accumulation of
 * poly.BuildGrandProductMixed (internal/poly/iop_utils.go:170-192,316-323)
 * after its numerator and denominator expressions are evaluated. */
int lg_grand_product(lg_ctx* ctx, const uint32_t* num, const uint32_t* den, uint64_t n, uint32_t* out, int on_device);

/* Allocation-free grand product.  No counterpart in the reference: it is for
 * callers that cannot call cudaMalloc (a framework's caching allocator owns
 * the device memory, a memory-capped sandbox, a request path that must not
 * allocate).  Same result as lg_grand_product; num, den and out are DEVICE
 * pointers on the current device (n E6 rows, 6 words each), launched on
 * `cuda_stream` (a cudaStream_t; NULL = default stream) and not waited for.
 * Its only scratch is a fixed 96 KiB device array inside this library, held
 * by every GPU that loads it until the process exits: n above 2^22 rows
 * returns LG_ERR_UNSUPPORTED.  The first call on a device looks up that
 * array's address (make it before any stream capture); calls whose work
 * overlaps on the GPU share the array and race, so serialize them.  It calls
 * no cudaMalloc, cudaFree or other allocating routine.  An error already
 * pending on the calling thread is left in place and returns LG_ERR_CUDA
 * before anything is launched; its four launches count in
 * lg_kernel_launches(). */
int lg_grand_product_noalloc(const uint32_t* num, const uint32_t* den, uint64_t n, uint32_t* out, void* cuda_stream);

/* Measurement hooks (no counterpart in the reference, which times phases
 * with wall-clock callbacks, prover/prover.go:99-108): CUDA events recorded
 * on the context's stream.  lg_timer_mark records event `slot` (< 16);
 * lg_timer_elapsed waits for `to` and returns the milliseconds between the
 * two marks. */
int lg_timer_mark(lg_ctx* ctx, uint32_t slot);
int lg_timer_elapsed(lg_ctx* ctx, uint32_t from, uint32_t to, float* ms);
/* Number of kernels this library has launched since it was loaded. */
uint64_t lg_kernel_launches(void);
/* Number of constraint kernels compiled at run time (tuning "quotient_jit")
 * that this process holds, over all devices. */
uint64_t lg_jit_kernels(void);
/* Per-kernel event profiler: enable (1) clears and starts recording events
 * around the main kernels; lg_profile_report writes a JSON object
 * {kernel: {launches, ms, bytes, perms}} with algorithmic bytes and Poseidon2
 * permutations per kernel, plus "phases" (host milliseconds per prove
 * phase), "kernels_by_phase" and "timeline": one [kernel, phase index,
 * start ms, duration ms] per recorded launch, starts relative to the first
 * recorded launch, so gaps between launches show where the device waited. */
int lg_profile(lg_ctx* ctx, int enable);
int lg_profile_report(lg_ctx* ctx, char* buf, size_t* len);

#ifdef __cplusplus
}
#endif

#endif /* LOOM_GPU_H */
