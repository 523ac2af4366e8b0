/*
 * ltg.h -- C ABI of the B200 block-tensor contraction path.
 *
 * This is the drop-in boundary for libtensor's block-sparse contraction hot
 * path.  Each entry point replaces one reference interface (cited per
 * function).  Conventions:
 *   - every function returns an int status: LTG_OK (0) or an LTG_ERR_* code;
 *     ltg_last_error() gives a message for the calling thread;
 *   - no C++ exceptions cross this boundary;
 *   - handles are opaque; plain pointers and sizes only;
 *   - permutations use the reference's convention (libtensor/core/permutation.h):
 *     perm[i] is the position in the source sequence of the element that lands
 *     at position i;
 *   - one CUDA stream per context; calls are asynchronous on that stream
 *     unless stated otherwise; ltg_ctx_synchronize() waits for it.
 */
#ifndef LTG_H
#define LTG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    LTG_OK = 0,
    LTG_ERR_BAD_ARG = 1,
    LTG_ERR_BAD_DIMS = 2,        /* libtensor::bad_dimensions */
    LTG_ERR_SYMMETRY = 3,        /* libtensor::symmetry_violation / bad_symmetry */
    LTG_ERR_UNSUPPORTED = 4,
    LTG_ERR_OOM = 5,
    LTG_ERR_CUDA = 6,
    LTG_ERR_TIMEOUT = 7,         /* a bounded device wait gave up */
    LTG_ERR_STATE = 8
};

/* Contraction arithmetic (ltg_contract2 mode). */
enum {
    LTG_MODE_PLAIN_FP64 = 0,     /* FP64 DMMA tensor-core contraction (drop-in) */
    LTG_MODE_OZAKI_BF16 = 1,     /* split-precision: BF16 slices, FP32 accumulate */
    LTG_MODE_OZAKI_FP8 = 2,      /* split-precision: FP8 E4M3 slices, FP32 accumulate */
    LTG_MODE_OZAKI_INT8 = 3,     /* split-precision: INT8 slices, INT32 accumulate */
    LTG_MODE_OZAKI_CRT = 4       /* split-precision: INT8 residues modulo nslices (8..16,
                                    default 13) coprime moduli, INT32 accumulate,
                                    Chinese-remainder recombination in FP64 */
};

typedef struct ltg_ctx ltg_ctx;
typedef struct ltg_bt ltg_bt;
typedef struct ltg_plan ltg_plan;
typedef struct ltg_graph ltg_graph;

/* Block tensor description: block index space plus symmetry.
 * Symmetry elements are applied in the order perm, part, label (the order in
 * which libtensor::symmetry<N,T>::insert() receives them).                  */
typedef struct ltg_bt_spec {
    int32_t order;                  /* 1..8 */
    const int64_t *dims;            /* [order] extents */
    const int32_t *nsplit;          /* [order] number of split points per dim */
    const int64_t *splits;          /* concatenated split positions */
    /* se_perm generators (libtensor/symmetry/se_perm.h:28) */
    int32_t nperm;
    const int32_t *perm;            /* [nperm*order] */
    const double *perm_coeff;       /* [nperm] +1 symmetric, -1 antisymmetric */
    /* se_part (libtensor/symmetry/se_part.h:32), forbidden partitions only */
    int32_t has_part;
    const int64_t *part_pdims;      /* [order] partitions per dim (1 = none) */
    int64_t npart_forbidden;
    const int64_t *part_forbidden;  /* [npart_forbidden*order] partition indices */
    /* se_label (libtensor/symmetry/se_label.h:37) for abelian (XOR) tables */
    int32_t has_label;
    int32_t label_nirrep;           /* 1, 2, 4 or 8 */
    const int32_t *labels;          /* concatenated per-dim block labels, -1 = none */
    int32_t label_nintr;
    const int32_t *label_intr;      /* allowed intrinsic labels (OR) */
} ltg_bt_spec;

const char *ltg_last_error(void);
int ltg_version(void);

/* ---- context --------------------------------------------------------- */
int ltg_ctx_create(int device, ltg_ctx **out);
int ltg_ctx_destroy(ltg_ctx *ctx);
/* Waits for the context's stream.  Returns LTG_ERR_TIMEOUT (once) when a
 * bounded device wait of a split-precision products kernel gave up since the
 * last report; that call's results are invalid, the context stays usable. */
int ltg_ctx_synchronize(ltg_ctx *ctx);
/* Limit of one pipeline wait (mbarrier) inside the tcgen05 products kernels,
 * in nanoseconds of wall time; default 2e9 (2 s).  When a wait runs out, the
 * kernel stops its work, lets its bulk copies and MMAs in flight finish, frees
 * its tensor memory and returns; the host reports LTG_ERR_TIMEOUT.  0 means no
 * waiting at all (a wait whose phase has not completed at its first test gives
 * up), which makes the unwind path testable.  No reference counterpart (the
 * reference runs on the CPU and has no device waits). */
int ltg_ctx_set_wait_limit(ltg_ctx *ctx, uint64_t ns);
int ltg_ctx_wait_limit(ltg_ctx *ctx, uint64_t *ns);
/* Underlying cudaStream_t of the context (for event timing by callers). */
int ltg_ctx_stream(ltg_ctx *ctx, void **stream);
/* Host threads used for schedule construction (libutil::thread_pool role). */
int ltg_ctx_set_host_threads(ltg_ctx *ctx, int nthreads);
/* Number of device kernels launched by this context so far. */
int ltg_ctx_launch_count(ltg_ctx *ctx, int64_t *count);
/* Per-kernel device timing.  While enabled, every kernel launch of the
 * context (outside graph capture) is bracketed by CUDA events on its stream;
 * ltg_ctx_kernel_times() waits for the stream and returns, per kernel kind,
 * the summed device time (ms) and the number of timed launches since timing
 * was enabled.  Enabling resets the totals.  No reference counterpart (the
 * reference's libutil timers time host regions). */
enum {
    LTG_KERNEL_CONTRACT_FP64 = 0,   /* plain FP64 DMMA contraction */
    LTG_KERNEL_OZ_SPLIT = 1,        /* split-precision: FP64 -> slices */
    LTG_KERNEL_OZ_GEMM = 2,         /* split-precision: slice products */
    LTG_KERNEL_TRANSFER = 3,        /* btod_copy / btod_add */
    LTG_KERNEL_DOT = 4,             /* btod_dotprod (both passes) */
    LTG_KERNEL_SCALE = 5,
    LTG_KERNEL_FILL = 6,            /* seeded fill */
    LTG_KERNEL_DENOMINATOR = 7,
    LTG_KERNEL_OZ_COMBINE = 8,      /* split-precision: modular recombination */
    LTG_KERNEL_KINDS = 9
};
int ltg_ctx_set_timing(ltg_ctx *ctx, int32_t enable);
int ltg_ctx_kernel_times(ltg_ctx *ctx, double *ms, int64_t *launches);

/* ---- block tensors (libtensor/block_tensor/block_tensor.h:22) --------- */
int ltg_bt_create(ltg_ctx *ctx, const ltg_bt_spec *spec, ltg_bt **out);
/* New tensor with the block index space and symmetry of `a` permuted by
 * `perm` (so_permute; the result space of btod_copy(a, perm)). */
int ltg_bt_create_permuted(ltg_bt *a, const int32_t *perm, ltg_bt **out);
/* A block tensor for the sum of the terms P_t(a_t) (perms[t*order ..], NULL =
 * identities): the block index space of P_0(a_0) (all terms must have it) and
 * the symmetry every term has -- the permutational (anti)symmetry elements
 * common to all terms' groups, and the partition and label rules when all
 * terms carry the same ones (otherwise none, every block allowed).  The
 * intermediate of a sum in the letter interface; the reference derives the
 * symmetry of btod_add's result with so_dirsum/so_merge
 * (libtensor/gen_block_tensor/impl/gen_bto_add_impl.h:225-274), which this
 * never exceeds. */
int ltg_bt_create_sum_space(int32_t nterms, ltg_bt *const *a, const int32_t *perms, ltg_bt **out);
/* Symmetrizers (libtensor/block_tensor/btod_symmetrize2.h:19,
 * btod_symmetrize4.h:27) over a tensor: the symmetrizer's group S is
 * nidx = 2: {e, (i1 i2)} with idx = (i1, i2); nidx = -1: {e, P} with idx the
 * unitary permutation P (P P = e, e.g. a pair exchange); nidx = 4: the 24
 * permutations of the indexes idx[0..3].  Signs: +1 with symm, else -1 for
 * the exchange (the parity of the permutation for four indexes).
 * ltg_bt_create_symmetrized: a block tensor for S-sums of a: a's block index
 * space with S's generators, the elements of a's group that map S onto
 * itself, and a's partition and label rules if S leaves them unchanged.
 * ltg_symmetrize: b = c sum_{s in S} sign(s) P_s(a) (add: b += d c ...),
 * asynchronous on the context stream. */
int ltg_bt_create_symmetrized(ltg_bt *a, int32_t nidx, const int32_t *idx, int32_t symm, ltg_bt **out);
int ltg_symmetrize(ltg_bt *a, double c, int32_t nidx, const int32_t *idx, int32_t symm, ltg_bt *b,
                   int32_t add, double d);
/* A two-term symmetrizer fused into a contraction (btod_symmetrize2 over a
 * btod_contract2, libtensor/block_tensor/btod_symmetrize2.h:19,
 * gen_block_tensor/impl/gen_bto_symmetrize2_impl.h): r = c (T + sign P(T)),
 * T the plan's contraction with coefficients ka, kb, kc, S = {e, P} as in
 * ltg_symmetrize (nidx 2 or -1), in any mode: plain FP64, modular (nslices
 * moduli, 0: 13) or a slice mode at its default slice count (0, or 7 for
 * BF16 and INT8, 8 for FP8; other counts LTG_ERR_UNSUPPORTED).  The kernel
 * that writes T's elements -- the plain DMMA epilogue, the grouped products'
 * scatter, the modular recombination or the slice products' epilogue --
 * adds each of them straight into the canonical
 * blocks of r that its two terms reach (no temporary T); r is zeroed first,
 * so every element takes at most two adds and the result does not depend on
 * their order.  Assignment only (ltg_symmetrize over a formed T adds); r
 * must not be an operand of the contraction (LTG_ERR_UNSUPPORTED).
 * ltg_contract2_make_symmetrized: a tensor with the space of such sums (as
 * ltg_bt_create_symmetrized over the contraction's result). */
int ltg_contract2_make_symmetrized(ltg_plan *plan, int32_t nidx, const int32_t *idx, int32_t symm, ltg_bt **out);
int ltg_contract2_symmetrized(ltg_plan *plan, ltg_bt *r, int32_t mode, int32_t nslices, double c, int32_t nidx,
                              const int32_t *idx, int32_t symm, double ka, double kb, double kc);
int ltg_bt_destroy(ltg_bt *bt);
/* Canonical allowed blocks: count and packed arena size in elements. */
int ltg_bt_info(const ltg_bt *bt, int32_t *order, int64_t *nblocks, int64_t *nelems);
/* Per canonical block: absolute block index, arena offset, element count. */
int ltg_bt_blocks(const ltg_bt *bt, int64_t *abs_idx, int64_t *offset, int64_t *size);
/* Block-index dims (number of blocks per dimension). */
int ltg_bt_bidims(const ltg_bt *bt, int64_t *bidims);
/* Extents of the block with block index bidx
 * (block_index_space::get_block_dims). */
int ltg_bt_block_dims(const ltg_bt *bt, const int64_t *bidx, int64_t *dims);
/* Non-zero canonical blocks (req_nonzero_blocks,
 * gen_block_tensor/gen_block_tensor_ctrl.h:100). Returns the count in *n. */
int ltg_bt_nonzero(const ltg_bt *bt, int64_t *abs_idx, int64_t cap, int64_t *n);
/* Orbit of a block: canonical index, transform canonical->block, allowed
 * (libtensor/core/orbit.h). Returns allowed (0/1) in *allowed. */
int ltg_bt_orbit(const ltg_bt *bt, int64_t abs_idx, int64_t *canonical,
                 int32_t *perm, double *coeff, int32_t *allowed);
/* Whole-arena transfer of all canonical blocks in ltg_bt_blocks order
 * (synchronous).  Upload marks every block non-zero. */
int ltg_bt_upload(ltg_bt *bt, const double *host);
int ltg_bt_download(ltg_bt *bt, double *host);
/* Single-block transfer (req_block / ret_block). */
int ltg_bt_upload_block(ltg_bt *bt, const int64_t *bidx, const double *data);
int ltg_bt_download_block(ltg_bt *bt, const int64_t *bidx, double *data);
/* Asynchronous whole-arena transfer on the context stream (pinned host
 * memory recommended). */
int ltg_bt_upload_async(ltg_bt *bt, const double *host);
int ltg_bt_download_async(ltg_bt *bt, double *host);
/* Zero every block and mark all blocks zero (btod_set(0)). */
int ltg_bt_set_zero(ltg_bt *bt);
/* Mark all canonical blocks non-zero without touching data. */
int ltg_bt_mark_nonzero(ltg_bt *bt);
/* Make one canonical block zero (gen_block_tensor_ctrl::req_zero_block,
 * gen_block_tensor/gen_block_tensor_ctrl.h): its data is cleared and it
 * leaves the non-zero list. */
int ltg_bt_zero_block(ltg_bt *bt, const int64_t *bidx);
/* Device fill of all canonical blocks with the seeded, symmetrised test
 * distribution of ltg_seeded_value() (one launch). */
int ltg_bt_fill_seeded(ltg_bt *bt, uint64_t seed, double scale);
/* Host fill with bit-identical values (multi-threaded CPU). */
int ltg_bt_fill_seeded_host(const ltg_bt *bt, uint64_t seed, double scale, double *host);
/* Raw device pointer of the arena. */
int ltg_bt_device_ptr(ltg_bt *bt, double **ptr);

/* ---- btod_contract2 (libtensor/block_tensor/btod_contract2.h:29-140) -- */
/* Builds the contraction of a (order N+K) and b (order M+K): permc is the
 * result permutation (contraction2(permc)), pairs[2*K] the contracted index
 * pairs (contraction2::contract(ia, ib)).  Schedule construction runs here
 * (gen_bto_contract2::make_schedule). */
int ltg_contract2_create(ltg_ctx *ctx, int32_t n, int32_t m, int32_t k,
                         const int32_t *permc, const int32_t *pairs,
                         ltg_bt *a, ltg_bt *b, ltg_plan **out);
/* Schedules are cached process-wide: ltg_contract2_create with a contraction
 * and operands of a description seen before (block index spaces, symmetry
 * elements, non-zero blocks) reuses the earlier schedule instead of building
 * it again (the reference builds it in every btod_contract2 constructor,
 * libtensor/gen_block_tensor/impl/gen_bto_contract2_nzorb_impl.h:354-477).
 * Capacity in schedules (default 64, least recently used dropped; 0 turns
 * the cache off) and its hit/miss counts: */
int ltg_schedule_cache_set_capacity(int64_t entries);
int ltg_schedule_cache_stats(int64_t *hits, int64_t *misses, int64_t *entries);
/* Creates an empty result tensor with the derived block index space and
 * symmetry (btod_contract2::get_bis / get_symmetry). */
int ltg_contract2_make_result(ltg_plan *plan, ltg_bt **c);
/* Non-zero canonical C blocks (get_schedule). */
int ltg_plan_schedule(ltg_plan *plan, int64_t *abs_idx, int64_t cap, int64_t *n);
/* Coalesced pair list of schedule entry i: per pair
 * {aia, acia, perm_a[NA], coeff_a bits, aib, acib, perm_b[NB], coeff_b bits}
 * as int64 (coefficients as raw IEEE-754 bits). */
int ltg_plan_pairs(ltg_plan *plan, int64_t i, int64_t *out, int64_t cap, int64_t *npairs);
/* Algorithmic flops: sum over C blocks and pairs of 2*|C block|*K. */
int ltg_plan_flops(ltg_plan *plan, double *flops);
/* perform(): C = kc * contr(ka*A, kb*B) (add == 0), or C += d * ... (add).
 * nslices is the slice count of the split-precision modes (ignored by
 * LTG_MODE_PLAIN_FP64). */
int ltg_contract2(ltg_plan *plan, ltg_bt *c, int32_t mode, int32_t nslices,
                  double ka, double kb, double kc, int32_t add, double d);
/* Bytes the split pass(es) of a split-precision mode move for this call:
 * FP64 operand bytes read (twice for the modular mode: exponent and residue
 * passes) and slice/residue bytes written.  No reference counterpart (used
 * for rooflines). */
int ltg_contract2_split_bytes(ltg_plan *plan, ltg_bt *c, int32_t mode, int32_t nslices, double ka,
                              double kb, double kc, int32_t add, double d, int64_t *read_bytes,
                              int64_t *write_bytes);
int ltg_plan_destroy(ltg_plan *plan);
/* Forces one tile shape for every C block (cfg >= 0) or restores the
 * automatic choice (-1).  No reference counterpart: the reference hands each
 * block pair to BLAS. */
int ltg_contract2_set_tile(ltg_plan *plan, int32_t cfg);
/* Plain FP64 mode: k chunks per output tile.  0 (default) cuts the k range of
 * the last work items of a launch into 2-4 chunks when that evens out the end
 * of the launch; 1 never cuts; 2-4 cut every tile into that many chunks.  The
 * chunks' partial tiles are summed in k order by a second kernel, so results
 * do not depend on scheduling (they differ from the uncut sum in rounding
 * only).  No reference counterpart. */
int ltg_contract2_set_split_k(ltg_plan *plan, int32_t k);
/* Modular mode (LTG_MODE_OZAKI_CRT): enables (default) or disables grouped
 * products.  When no pair list was shortened by coalescing, C blocks whose row
 * blocks (C dims taken from A) and column blocks (C dims taken from B) are
 * linked by the schedule are computed as one product over the union of their
 * contracted blocks (operand cells that no pair uses stay zero), instead of one
 * product per C block and pair.  The integer products are exact, so both
 * forms give identical bits; grouping only changes the tile shapes (blocks of
 * a few rows, as under point-group symmetry, fill whole tiles).  No reference
 * counterpart. */
int ltg_contract2_set_grouping(ltg_plan *plan, int32_t enable);
/* Modular mode: the one-read split of row families -- panels whose rows feed
 * the same rows of C and nothing else does -- which forms each row's exact
 * exponent and its residues in one kernel (the second read of each tile hits
 * L2) instead of the exponent pass and the residue pass: shape 0 off
 * (default), 1 or 2 (rows per CTA, threads, CTAs per SM: 2/512/2, 2/256/4).
 * Identical bits to the two passes with exact exponents; on the ladder
 * o=40 v=240 slower than the two passes (2.68 ms for shape 2 against 2.40
 * with an exact exponent pass, 1.79 with sampled bounds).  No reference
 * counterpart. */
int ltg_contract2_set_fused_split(ltg_plan *plan, int32_t enable);
/* Modular mode: how the row exponents (the scale of each operand row) are
 * found.  1 (default): rows of at least 1024 k words read one 32-element run
 * in 16 for a bound one binade above the sampled maximum; the residue
 * pass forms their exact maxima while it reads them, and redoes the rows whose
 * bound was too small with the exact exponent -- so every row's integers stay
 * within 2^P, at most one bit of the P-bit operands is given up, and the
 * exponent pass reads about 1/16 of those operands.  0: an exponent pass
 * over every element (exact maxima).  Both give results within the mode's
 * error bound; their bits differ where the bound is a binade above the
 * maximum.  No reference counterpart. */
int ltg_contract2_set_crt_bound(ltg_plan *plan, int32_t sampled);
/* Modular mode: rows of the products kernel's work items, 256 (two MMA
 * tiles sharing each operand tile of the other side; also 0, the default) or
 * 128 (one MMA tile; the epilogue of one modulus overlaps the products of the
 * next, at twice the operand traffic per product).  Both give identical bits.
 * No reference counterpart. */
int ltg_contract2_set_crt_rows(ltg_plan *plan, int32_t rows);
/* Modular mode: 32-byte k blocks per pipeline stage of the products kernel
 * (2, 3, 4 (default) or 6; the stages fill about 200 KB of shared memory,
 * each stage's k blocks moved as one bulk copy per operand tile).  No
 * reference counterpart. */
int ltg_contract2_set_crt_stage(ltg_plan *plan, int32_t kblocks);
/* Host-side summary of the grouped products the modular mode would use for
 * result c: number of groups, C blocks they cover, flops of the grouped
 * products (padding of the contracted blocks to 4 included) and algorithmic
 * flops of the blocks they cover.  Needs no device.  Any pointer may be NULL. */
int ltg_contract2_group_info(ltg_plan *plan, ltg_bt *c, int64_t *ngroups, int64_t *nblocks,
                             double *grouped_flops, double *block_flops);
/* Autotuner: for every distinct C-block shape (M, N) of the plan, costliest
 * first, times each compiled tile shape on the real contraction (reps calls,
 * CUDA events) and keeps the fastest.  Overwrites c. */
int ltg_contract2_autotune(ltg_plan *plan, ltg_bt *c, int32_t mode, int32_t nslices,
                           double ka, double kb, double kc, int32_t reps);
/* Autotuned table: C-block shape -> tile shape index. */
int ltg_plan_tiles(ltg_plan *plan, int64_t *m, int64_t *n, int32_t *cfg, int64_t cap,
                   int64_t *count);

/* ---- caller-built task lists ------------------------------------------ */
/* One block-pair product C[c_off..] += coeff * A[a_off..] * B[b_off..] as
 * LTG_TASK_WORDS int64 (element offsets into the tensors' arenas):
 *   [0] c_off  [1] a_off  [2] b_off
 *   [3] nm, [4..15]  up to four (extent, stride in A, stride in C)   (m)
 *   [16] nn, [17..28] up to four (extent, stride in B, stride in C)  (n)
 *   [29] nk, [30..41] up to four (extent, stride in A, stride in B)  (k)
 *   [42] coeff as raw IEEE-754 bits.
 * This is the product list that gen_bto_contract2_block::compute_block
 * (libtensor/gen_block_tensor/impl/gen_bto_contract2_block_impl.h) hands to
 * the dense kernel, one entry per (C block, pair); the record layout itself
 * has no reference counterpart. */
#define LTG_TASK_WORDS 43
/* Writes the task list of plan for result c (coefficients ka = kb = kc = 1)
 * into tasks (cap entries), *ntasks = the full count. */
int ltg_plan_export_tasks(ltg_plan *plan, ltg_bt *c, int64_t *tasks, int64_t cap, int64_t *ntasks);
/* Plan from a caller-built task list over a and b.  Consecutive tasks with
 * the same c_off form one C block (same m and n extents; C strides from the
 * first); a C block's first task assigns or accumulates as ltg_contract2's
 * add says, the rest accumulate.  Runs in LTG_MODE_PLAIN_FP64 only; the
 * result tensor must hold every c_off range.  Free with ltg_plan_free. */
int ltg_plan_contract2_upload(ltg_ctx *ctx, ltg_bt *a, ltg_bt *b, const int64_t *tasks,
                              int64_t ntasks, ltg_plan **out);

/* ---- alternative names of the entry points above ----------------------- */
int ltg_bt_alloc(ltg_ctx *ctx, const ltg_bt_spec *spec, ltg_bt **out);      /* ltg_bt_create */
int ltg_bt_free(ltg_bt *bt);                                                /* ltg_bt_destroy */
int ltg_bt_upload_blocks(ltg_bt *bt, const double *host);                   /* ltg_bt_upload */
int ltg_bt_download_blocks(ltg_bt *bt, double *host);                       /* ltg_bt_download */
int ltg_plan_free(ltg_plan *plan);                                          /* ltg_plan_destroy */
int ltg_copy_perm(ltg_bt *a, const int32_t *perm, double c, ltg_bt *b,      /* ltg_copy */
                  int32_t add, double d);
int ltg_add_perm_n(int32_t nterms, ltg_bt *const *a, const int32_t *perms,  /* ltg_add */
                   const double *coeffs, ltg_bt *b, int32_t add, double d);
const char *ltg_last_error_string(void);                                    /* ltg_last_error */

/* ---- btod_copy / btod_add / btod_dotprod ------------------------------ */
/* b = c * perm(a)  or  b += d * c * perm(a)   (btod_copy.h:38-115) */
int ltg_copy(ltg_bt *a, const int32_t *perm, double c, ltg_bt *b,
             int32_t add, double d);
/* b = sum_t c_t * perm_t(a_t)  or  b += d * sum ...  (btod_add.h:38-131) */
int ltg_add(int32_t nterms, ltg_bt *const *a, const int32_t *perms,
            const double *coeffs, ltg_bt *b, int32_t add, double d);
/* <perma(a), permb(b)> over the full tensor (btod_dotprod.h:35-70);
 * synchronous, result in *out. */
int ltg_dotprod(ltg_bt *a, const int32_t *perma, ltg_bt *b,
                const int32_t *permb, double *out);
/* Asynchronous form: result left in device memory at *dev_out. */
int ltg_dotprod_async(ltg_bt *a, const int32_t *perma, ltg_bt *b,
                      const int32_t *permb, double *dev_out);
/* Allocation-free dot product sum_i x[i]*y[i] of two device arrays of the
 * calling thread's current device, run on `stream` (a cudaStream_t; NULL =
 * default stream); synchronous, result in *out (host).  No reference
 * counterpart: it serves callers that must not allocate device memory (error
 * paths after an out-of-memory failure, programs whose memory is reserved by
 * another allocator, loops that cudaMalloc/cudaFree would stall).  Partial
 * sums live in one fixed device array per device (16384 partials of 65536
 * elements each): n is limited to 2^30 elements and larger n returns
 * LTG_ERR_BAD_ARG.  All calls on a device share that array, so calls that
 * overlap in time race and must be serialised by the caller.  The first call
 * on a device is not allocation-free: it loads the library's module for this
 * entry point (device memory for the array and the kernels) and looks up the
 * array's address.  Make one call with n > 0 early on each device, while
 * memory is free and before any stream capture on it; later calls allocate
 * nothing.  Not usable after cudaDeviceReset.  The sum order depends only
 * on n. */
int ltg_dot_noalloc(const double *x, const double *y, int64_t n, void *stream,
                    double *out);
/* a *= c  (btod_scale) */
int ltg_scale(ltg_bt *a, double c);
/* a[i,j,a,b] /= (e_i + e_j - e_a - e_b) style denominator over a 4-index
 * tensor: divides every element by (sum of eps over the index positions with
 * sign +1 for the first `nocc` dims and -1 for the rest).  eps is a host array
 * per dim concatenated (dims[0]+...+dims[3]); it is kept on the device, so a
 * repeated call with the same eps (also inside a graph capture) only launches.
 * Asynchronous on the context stream. */
int ltg_denominator(ltg_bt *a, const double *eps_host, int32_t nocc);

/* ---- CUDA graphs over a context's stream ------------------------------ */
int ltg_graph_begin(ltg_ctx *ctx);
int ltg_graph_end(ltg_ctx *ctx, ltg_graph **out);
int ltg_graph_launch(ltg_graph *g);
int ltg_graph_destroy(ltg_graph *g);

#ifdef __cplusplus
}
#endif

#endif /* LTG_H */
