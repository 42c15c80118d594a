/*
 * hlrc.h — C ABI of the B200 H-matrix / uniform-H matrix-vector product.
 *
 * The product computes   y := y + alpha * op(M) * x   for an H-matrix M
 * (dense leaves and low-rank leaves U*V^T) or a uniform-H matrix M (shared,
 * non-nested row/column cluster bases with coupling matrices), exactly like
 * HLR's CPU paths:
 *
 *   hlr::tbb::mul_vec(alpha, op_M, M, x, y)              include/hlr/tbb/arith.hh:312-340
 *   hlr::seq::mul_vec / hlr::mul_vec                     include/hlr/arith/mulvec.hh:27-81
 *   hlr::tbb::uniform::mul_vec(alpha, op_M, M, x, y,
 *                              rowcb, colcb)             include/hlr/tbb/arith_uniform.hh:36-96
 *
 * Indices are in the matrix's internal (cluster-tree permuted) order, as in
 * HLR, where the coefficient function is wrapped in TPermCoeffFn
 * (programs/mvm/mvm.hh:66).
 *
 * Conventions
 *  - Every entry point returns an hlrc_status; no C++ exception crosses the
 *    ABI.  hlrc_last_error() returns a message for the calling thread.
 *  - Matrices are column-major; low-rank leaves store M = U * V^T with
 *    U (nrows x rank) and V (ncols x rank), as hlr::matrix::lrmatrix
 *    (include/hlr/matrix/lrmatrix.hh:39-204).
 *  - y is accumulated (y += ...), never overwritten; alpha == 0 is a no-op,
 *    as in hlr::tbb::mul_vec (include/hlr/tbb/arith.hh:54-55).
 *  - A device handle is immutable after upload.  Each handle owns one
 *    scratch workspace, used by hlrc_mvm and hlrc_mvm_host, so two hlrc_mvm
 *    calls on the same handle must be ordered on one stream.  Concurrent
 *    products on one handle (several streams, several host threads) each
 *    pass their own hlrc_workspace to hlrc_mvm_ws.  The host API is
 *    thread-safe except for hlrc_free / hlrc_workspace_free of an object in
 *    use and hlrc_set_tuning / hlrc_set_profiling during products.
 *  - Device pointers (x, y) are plain CUDA device pointers; `stream` is a
 *    cudaStream_t passed as void* (NULL = legacy default stream).
 *
 * Nothing here takes or returns a torch type.
 */
#ifndef HLRC_H
#define HLRC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HLRC_ABI_VERSION 1

/* ------------------------------------------------------------------ status */
typedef enum hlrc_status {
    HLRC_OK                 = 0,
    HLRC_ERR_ARG            = 1,  /* null pointer / bad argument            */
    HLRC_ERR_SHAPE          = 2,  /* inconsistent sizes, bad block layout    */
    HLRC_ERR_OOM            = 3,  /* device or host allocation failed        */
    HLRC_ERR_CUDA           = 4,  /* a CUDA runtime call failed              */
    HLRC_ERR_TIMEOUT        = 5,  /* a bounded device wait gave up           */
    HLRC_ERR_UNSUPPORTED_OP = 6,  /* op not supported for this matrix kind   */
    HLRC_ERR_NOT_CONVERGED  = 7,  /* iterative solver hit its iteration cap  */
    HLRC_ERR_INTERNAL       = 8
} hlrc_status;

/* matop_t of HLIBpro (apply_normal/transposed/adjoint); for real data the
 * transposed and adjoint products are identical. */
typedef enum hlrc_op {
    HLRC_OP_N = 0,   /* apply_normal     */
    HLRC_OP_T = 1,   /* apply_transposed */
    HLRC_OP_C = 2    /* apply_adjoint    */
} hlrc_op;

/* Storage precision of the device copy of the matrix data.
 * Vectors x, y are always FP64; the per-row-tile accumulation of y is FP64. */
typedef enum hlrc_precision {
    HLRC_PREC_F64  = 0,  /* FP64 storage, FP64 arithmetic (drop-in path)        */
    HLRC_PREC_F32  = 1,  /* FP32 storage, FP32 products, FP64 y accumulation     */
    HLRC_PREC_BF16 = 2,  /* BF16 storage, per-column FP32 scale, FP32 products   */
    HLRC_PREC_F16  = 3,  /* FP16 storage, per-column FP32 scale, FP32 products   */
    HLRC_PREC_MIXED = 4, /* per-column choice FP32/FP16 from the singular values
                            (HLR's VALR rule, include/hlr/compress/valr.hh:402-510);
                            dense leaves FP32                                    */
    HLRC_PREC_BFP = 5    /* block floating point, byte-aligned: VALR tolerances
                            u_i as for MIXED; a column whose bit rate
                            ceil(-log2 u_i) (HLR's BFP rule,
                            include/hlr/compress/bfp.hh:79-80) is at most 15 is
                            stored as 16-bit integers, every other column and
                            the dense leaves as 24-bit integers (22 bits of
                            magnitude), each chunk with a power-of-two scale.
                            One-vector kernels only: multi-vector products
                            loop them                                          */
} hlrc_precision;

/* ---------------------------------------------------------- host structures
 * A caller describes its matrix by a flat list of leaf blocks.  The list
 * order is the order in which the CPU reference visits leaves
 * (hlr::mul_vec recursion, block row i then block column j).
 */
typedef enum hlrc_leaf_kind {
    HLRC_LEAF_DENSE   = 0,   /* hlr::matrix::dense_matrix  (dense_matrix.hh:36)   */
    HLRC_LEAF_LOWRANK = 1    /* hlr::matrix::lrmatrix      (lrmatrix.hh:39)       */
} hlrc_leaf_kind;

typedef struct hlrc_block {
    int64_t       row0, nrows;   /* row index set [row0, row0+nrows)          */
    int64_t       col0, ncols;   /* column index set [col0, col0+ncols)       */
    int32_t       kind;          /* hlrc_leaf_kind                            */
    int32_t       rank;          /* low-rank: k (may be 0)                    */
    const double* D;             /* dense: nrows x ncols, column-major        */
    int64_t       ldd;
    const double* U;             /* low-rank: nrows x rank                     */
    int64_t       ldu;
    const double* V;             /* low-rank: ncols x rank;  M = U * V^T       */
    int64_t       ldv;
    const double* sv;            /* optional: rank singular values (descending)
                                    of the block, used by HLRC_PREC_MIXED; NULL
                                    = derive from ||U(:,i)||*||V(:,i)||        */
} hlrc_block;

typedef struct hlrc_h_desc {
    int64_t            nrows, ncols;
    int64_t            nblocks;
    const hlrc_block*  blocks;
} hlrc_h_desc;

/* uniform-H: shared_cluster_basis (shared_cluster_basis.hh:39-356) per
 * cluster, uniform_lrmatrix (uniform_lrmatrix.hh:59-154) per admissible leaf */
typedef struct hlrc_basis {
    int64_t       ofs, size;     /* cluster index set [ofs, ofs+size)          */
    int32_t       rank;          /* k_t (0 allowed)                           */
    int32_t       pad_;
    const double* V;             /* size x rank, column-major                  */
    int64_t       ldv;
} hlrc_basis;

typedef struct hlrc_uniform_block {
    int64_t       row0, nrows, col0, ncols;
    int32_t       kind;          /* HLRC_LEAF_DENSE or HLRC_LEAF_LOWRANK        */
    int32_t       row_basis;     /* low-rank: index into row_bases            */
    int32_t       col_basis;     /* low-rank: index into col_bases            */
    int32_t       pad_;
    const double* S;             /* low-rank: k_row x k_col coupling, col-major */
    int64_t       lds;
    const double* D;             /* dense: nrows x ncols                       */
    int64_t       ldd;
} hlrc_uniform_block;

typedef struct hlrc_uniform_desc {
    int64_t                    nrows, ncols;
    int64_t                    nrow_bases;
    const hlrc_basis*          row_bases;
    int64_t                    ncol_bases;
    const hlrc_basis*          col_bases;
    int64_t                    nblocks;
    const hlrc_uniform_block*  blocks;
} hlrc_uniform_desc;

/* H^2 matrix (nested cluster bases), the structure of HLR's
 * nested_cluster_basis (include/hlr/matrix/nested_cluster_basis.hh) and its
 * product (include/hlr/arith/h2.hh:21-40, arith/detail/h2.hh:238-330): a
 * cluster tree per side, an explicit basis V (size x rank) at the leaves,
 * and for every non-root cluster the transfer matrix E (rank x rank of the
 * parent) with V_parent = [V_son0 E_son0; V_son1 E_son1].  Blocks are
 * hlrc_uniform_block entries whose row_basis / col_basis index the
 * clusters; a low-rank block (t, s) is V_t S W_s^T.                          */
typedef struct hlrc_h2_cluster {
    int64_t       ofs, size;     /* index set                                   */
    int32_t       son[2];        /* child clusters, -1 for none                 */
    int32_t       parent;        /* -1 for the root                             */
    int32_t       rank;
    const double* V;             /* leaves: size x rank, col-major               */
    int64_t       ldv;
    const double* E;             /* non-root: rank x parent rank, col-major      */
    int64_t       lde;
} hlrc_h2_cluster;

typedef struct hlrc_h2_desc {
    int64_t                    nrows, ncols;
    int64_t                    nrow_clusters;
    const hlrc_h2_cluster*     row_clusters;
    int64_t                    ncol_clusters;
    const hlrc_h2_cluster*     col_clusters;
    int64_t                    nblocks;
    const hlrc_uniform_block*  blocks;
} hlrc_h2_desc;

typedef struct hlrc_options {
    int32_t precision;     /* hlrc_precision (default HLRC_PREC_F64)            */
    int32_t max_nrhs;      /* workspace sized for this many right-hand sides   */
    double  mixed_eps;     /* HLRC_PREC_MIXED: target accuracy (e.g. 1e-6)      */
    int32_t device;        /* CUDA device ordinal (-1 = current)                */
    /* plan-level choices (0 = default), picked by hlr_b200.tune.autotune_plan:
     * finish_slots: outputs of the tile T-form with more tile partials than
     *   this are summed in two levels (2..64, default 16);
     * piece_tiles: column clusters of the 64-vector T-form longer than this
     *   many tiles are cut into pieces summed by a finish (1..32, default 32) */
    int32_t finish_slots;
    int32_t piece_tiles;
    /* 1: the descriptor's leaf data (D, U, V, sv) is in device memory of this
     * device (an on_device build); FP64 stores are filled on the device,
     * other precisions copy the leaves to the host first                   */
    int32_t leaves_on_device;
    /* near_field (products of op N): 1 = the dense leaves' D x is summed in
     * the last pass with the low-rank part (as HLR's mul_vec sums every
     * block of a row, tbb/detail/arith.hh:95-124); 2 = D x is its own pass,
     * launched on a side stream at the start of the product and joined
     * before the pass that adds the low-rank part to y, so that it overlaps
     * the dependent low-rank passes, in one- and 8-vector products; 0 =
     * default: 2 for one-vector products, 1 for multi-vector ones (their
     * passes are compute-heavy: nothing to overlap).  With 2, D x is added
     * first, then the low-rank part, per row tile; the 64-vector product of
     * 16-bit stores always takes the fused pass.                          */
    int32_t near_field;
    int32_t reserved[3];
} hlrc_options;

/* accounting of one product, following HLR's mul_vec_flops /
 * mul_vec_datasize (arith/mulvec.hh:795-874, arith/uniform.hh:285-325) */
typedef struct hlrc_info {
    int64_t n_rows, n_cols;
    int64_t n_dense, n_lowrank;        /* leaves                                */
    int64_t n_row_tiles, n_col_tiles;  /* <=64-row output tiles of y            */
    int64_t matrix_bytes;              /* stored matrix bytes on the device     */
    int64_t algorithmic_bytes;         /* matrix bytes + vector bytes, 1 rhs    */
    int64_t flops;                     /* per product, 1 rhs                    */
    int64_t workspace_bytes;
    int64_t device_bytes;              /* all device memory owned by the handle */
    int32_t precision;
    int32_t kind;                      /* 0 = H, 1 = uniform-H                  */
    int32_t max_rank;
    int32_t launches[3];               /* kernel launches per product, op N/T/C
                                          (0 = op unsupported)                  */
    int64_t scratch_bytes;             /* scratch of one one-vector product:
                                          low-rank coefficients and per-tile
                                          partial sums (what hlrc_mvm_noalloc
                                          takes from its static array)          */
} hlrc_info;

typedef struct hlrc_hmat_s* hlrc_hmat;

/* ------------------------------------------------------------ core entry points */

/* Returns HLRC_ABI_VERSION. */
int         hlrc_abi_version(void);

/* Message of the last failing call on this thread ("" if none). */
const char* hlrc_last_error(void);

void        hlrc_default_options(hlrc_options* opts);

/* Flatten an H-matrix into the device layout and upload it.
 * Replaces nothing on the HLR side, which multiplies its Hpro::TMatrix tree
 * in place: the caller walks that tree in hlr::mul_vec's recursion order
 * (arith/mulvec.hh:38-60) and fills one hlrc_block per leaf, pointing at the
 * leaf's own column-major arrays (dense_matrix::mat(), lrmatrix::U() / V()). */
hlrc_status hlrc_upload_h(const hlrc_h_desc* desc, const hlrc_options* opts,
                          hlrc_hmat* out);

/* Batch of `count` H-matrices as one handle: member i occupies rows and
 * columns [offsets[i], offsets[i] + n_i) of a block-diagonal matrix of size
 * offsets[count] (offsets may leave gaps, e.g. to pad every member to the
 * same length).  Every pass of the product then runs as one launch over the
 * blocks of all members, so x and y are the concatenations of the members'
 * vectors.  No counterpart in the reference (which multiplies one matrix
 * per call); each member is checked like hlrc_upload_h.                     */
hlrc_status hlrc_upload_h_batch(const hlrc_h_desc* descs, int count,
                                const int64_t* offsets,
                                const hlrc_options* opts, hlrc_hmat* out);

/* Same for a uniform-H matrix (row/column cluster bases + couplings).        */
hlrc_status hlrc_upload_uniform(const hlrc_uniform_desc* desc,
                                const hlrc_options* opts, hlrc_hmat* out);

/* Same for an H^2 matrix (nested cluster bases).  Replaces the H^2 product
 * hlr::h2::mul_vec(alpha, op, M, x, y, rowcb, colcb) (arith/h2.hh:21-40):
 * op N runs the forward transform (leaf bases, then transfer matrices level
 * by level up the column tree), the couplings, the backward transform (level
 * by level down the row tree, then the leaf bases) and the near field;
 * op C the same with the roles of the trees exchanged.  op T is rejected
 * (HLRC_ERR_UNSUPPORTED_OP), as for uniform-H.  FP64 only.                  */
hlrc_status hlrc_upload_h2(const hlrc_h2_desc* desc, const hlrc_options* opts, hlrc_hmat* out);

/* Dry run of hlrc_upload_h / hlrc_upload_uniform: validates the descriptor,
 * flattens it on the host and reports the accounting and the device
 * footprint that an upload would need, without touching a GPU.  Lets a
 * caller size device memory before committing (no reference counterpart;
 * the numbers follow mul_vec_flops / mul_vec_datasize).                     */
hlrc_status hlrc_plan_info_h(const hlrc_h_desc* desc, const hlrc_options* opts,
                             hlrc_info* info);
hlrc_status hlrc_plan_info_uniform(const hlrc_uniform_desc* desc,
                                   const hlrc_options* opts, hlrc_info* info);
hlrc_status hlrc_plan_info_h2(const hlrc_h2_desc* desc, const hlrc_options* opts, hlrc_info* info);

/* Row partition of an H-matrix for one product shared by `parts` processes
 * (one per GPU): cuts[0] = 0 <= cuts[1] <= ... <= cuts[parts] = nrows (cuts
 * holds parts + 1 entries), no leaf straddles a cut, and the leaves between
 * consecutive cuts hold about equal stored bytes.  Rank r then uploads the
 * leaves of rows [cuts[r], cuts[r+1]) as an (rows x ncols) H-matrix, rows
 * shifted by -cuts[r], and owns those entries of x and y: op N all-gathers
 * x before its product, op T / C sums the ranks' full-length results (the
 * per-cluster ownership of y in HLR's mul_vec_cl, tbb/detail/arith.hh:
 * 406-448, spread over processes).  Host only.                              */
hlrc_status hlrc_row_cuts(const hlrc_h_desc* desc, int parts, int64_t* cuts);

/* y := y + alpha * op(M) * x on `stream`.
 * x: ncols(op) x nrhs device array (leading dimension ldx),
 * y: nrows(op) x nrhs device array (leading dimension ldy).
 * Replaces hlr::tbb::mul_vec (tbb/arith.hh:312-340) for H-matrices and
 * hlr::tbb::uniform::mul_vec (tbb/arith_uniform.hh:36-96) for uniform-H.
 * Uniform-H supports op N and C only; op T returns HLRC_ERR_UNSUPPORTED_OP,
 * as uniform_lrmatrix::uni_apply_add asserts (uniform_lrmatrix.hh:473-513). */
hlrc_status hlrc_mvm(hlrc_hmat M, double alpha, int op, const double* x,
                     double* y, int nrhs, int64_t ldx, int64_t ldy,
                     void* stream);

/* Same with x, y in host memory: copies x and y to the device, runs the
 * product, copies y back, synchronises.  Matches the reference's call on
 * host-resident scalar_vectors.  Uses the handle's staging buffers and
 * workspace under a per-handle lock, so concurrent host calls on one handle
 * are correct but run one after the other.                                   */
hlrc_status hlrc_mvm_host(hlrc_hmat M, double alpha, int op, const double* x,
                          double* y, int nrhs, int64_t ldx, int64_t ldy);

/* y := y + alpha * op(M) * x for one right-hand side, without allocating.
 * No counterpart in the reference: HLR's products allocate temporaries on
 * every call.  Meant for callers that must not allocate device memory while
 * they run: code that executes while a stream capture in global mode is open
 * in the process (cudaMalloc/cudaFree are then illegal and break the
 * capture), latency-critical loops that cannot afford the device-wide
 * synchronisation cudaFree implies, and processes where another framework's
 * caching allocator has already reserved the device memory so that a new
 * cudaMalloc would fail.  The product runs the same kernels as hlrc_mvm, but
 * its scratch (low-rank coefficients and per-tile partial sums) comes from
 * one static 8 MiB device array in the library instead of the handle's
 * workspace; the call itself never calls cudaMalloc, cudaFree or any
 * allocating routine.
 *  - Limit: a matrix whose scratch exceeds 8 MiB (about 1M doubles: the sum
 *    of the low-rank ranks plus the partial sums of blocks spanning several
 *    tiles) is rejected with HLRC_ERR_SHAPE; use hlrc_mvm for it.
 *  - The first call on each device looks up the array's device address
 *    (cudaGetSymbolAddress, with that device current); make that first call
 *    before any stream capture.
 *  - Every call on a device shares the one array, which keeps the last
 *    call's contents (each call writes every entry before reading it).  Calls
 *    that overlap on the GPU — on different streams, or with different
 *    handles on the same device — race; order them on one stream.
 *  - Uniform-H and H^2 handles are accepted (op N and C).
 *  - A near field planned as its own pass (hlrc_options.near_field) runs
 *    first on `stream`, not beside the other passes: the same kernels in
 *    the same order on y, so the same result as hlrc_mvm.               */
hlrc_status hlrc_mvm_noalloc(hlrc_hmat M, double alpha, int op,
                             const double* x, double* y, void* stream);

hlrc_status hlrc_get_info(hlrc_hmat M, hlrc_info* info);

/* Caller-owned scratch for concurrent products on one handle.
 * HLR's TBB product may be called concurrently on one matrix with different
 * y (include/hlr/tbb/arith.hh:312-323; y is updated under per-chunk locks,
 * tbb/detail/arith.hh:95-124).  Here a handle is immutable and all scratch a
 * product writes lives in a workspace, so products of one handle on several
 * streams (or host threads) run concurrently when each passes its own
 * workspace; products that share a workspace must be ordered on one stream.
 *   hlrc_workspace_create: device scratch sized for M (one-vector products,
 *     and with max_nrhs > 1 the multi-vector kernels' blocks as well; a
 *     multi-vector product on a workspace without them loops one-vector
 *     products).  Allocates with cudaMalloc on M's device.
 *   hlrc_mvm_ws: hlrc_mvm with the workspace's scratch instead of the
 *     handle's; same arguments, results and status codes.  A workspace fits
 *     any handle on the same device whose scratch is not larger (typically
 *     the handle it was created for); otherwise HLRC_ERR_SHAPE.  Products on
 *     a workspace are not recorded by hlrc_set_profiling.
 *   hlrc_workspace_free: releases it (after the products using it ended).  */
typedef struct hlrc_workspace_s* hlrc_workspace;
hlrc_status hlrc_workspace_create(hlrc_hmat M, int max_nrhs, hlrc_workspace* out);
hlrc_status hlrc_mvm_ws(hlrc_hmat M, hlrc_workspace ws, double alpha, int op, const double* x, double* y,
                        int nrhs, int64_t ldx, int64_t ldy, void* stream);
hlrc_status hlrc_workspace_free(hlrc_workspace ws);

/* Launch shapes of a handle's products, chosen per matrix and device by the
 * autotuner (hlr_b200.tune.autotune times the candidates and caches the
 * winner).  No counterpart in the reference, whose TBB products have no
 * launch shapes; every setting computes the same product (the order of the
 * per-warp partial sums differs, so results agree to rounding).
 *   nform_warps, ttform_warps: warps per CTA (4, 8 or 16) of the one-vector
 *     N-form and tile T-form kernels (16 for small matrices, where each
 *     output tile's chain of loads sets the time);
 *   mr_min_nrhs: products with at least this many vectors use the
 *     8-vector tensor-core kernels, smaller ones loop the one-vector kernels
 *     (2..HLRC_MR_NEVER; HLRC_MR_NEVER always loops);
 *   wide_min_nrhs: op N products of FP16 / BF16 H-matrix handles uploaded
 *     with max_nrhs > 8 with at least this many vectors run the one-pass
 *     kernels on the tcgen05 tensor cores, 64 vectors per pass of the
 *     matrix; smaller ones use the 8-vector kernels (2..HLRC_MR_NEVER);
 *   overlap: 1 launches the one-vector kernels with programmatic dependent
 *     launch (each may be scheduled while its predecessor in the stream
 *     still runs and waits for it on the device before touching vectors),
 *     0 launches them plainly; the results are the same.
 * Defaults: 8, 8, 2, 9, 1.  hlrc_set_tuning rejects other values
 * (HLRC_ERR_ARG) and must not race with products of the same handle.      */
#define HLRC_MR_NEVER 1000000
typedef struct hlrc_tuning {
    int32_t nform_warps;
    int32_t ttform_warps;
    int32_t mr_min_nrhs;
    int32_t wide_min_nrhs;
    int32_t overlap;
    /* products with the near field on a side stream (hlrc_options.near_field):
     * the side pass is forked after this many of the other passes have been
     * launched (0 = at the start; 0..16, clamped to the pass that adds the
     * low-rank part to y).  Results do not depend on it.                   */
    int32_t side_at;
    int32_t reserved[2];
} hlrc_tuning;

hlrc_status hlrc_get_tuning(hlrc_hmat M, hlrc_tuning* t);
hlrc_status hlrc_set_tuning(hlrc_hmat M, const hlrc_tuning* t);

/* Device timing of the passes of the products (for roofline reporting).
 * While profiling is enabled every pass of every hlrc_mvm call is bracketed
 * by CUDA events on the call's stream.  hlrc_last_profile synchronises on
 * those events and returns, per pass *name* (static strings), the number of
 * launches, the summed milliseconds and the algorithmic bytes of one launch
 * (stored matrix bytes without padding, plus vector reads/writes), then
 * clears the records.  Returns the number of names written.  Products
 * captured into a CUDA graph with profiling enabled record their events as
 * external event-record nodes: after a replay, hlrc_last_profile returns
 * that replay's pass times (read it before the next replay).                */
hlrc_status hlrc_set_profiling(hlrc_hmat M, int enable);
int         hlrc_last_profile(hlrc_hmat M, const char** names, int* count,
                              double* ms, int64_t* bytes, int cap);

/* Number of kernels this handle has launched since upload (all entry
 * points); lets a caller count the launches inside a timed region.         */
int64_t     hlrc_launch_count(hlrc_hmat M);

hlrc_status hlrc_free(hlrc_hmat M);

/* Measured FP64 tensor-core (DMMA) throughput of `device` (-1 = current),
 * in TFLOP/s: a register-resident loop of m8n8k4 f64 MMAs timed with CUDA
 * events.  The compute roof of FP64 products with several right-hand sides,
 * reported beside the HBM roof.  No counterpart in the reference; changes
 * no device setting.                                                         */
hlrc_status hlrc_fp64_peak(int device, double* tflops);

/* Reads and clears the handle's device error word (synchronous).  Kernels
 * that wait with a bound set it when a wait runs out; the products launched
 * since then are incomplete.  0 means no error; bit 0 (value 1): a copy wait
 * of an H^2 tree sweep ran out; bit 1 (value 2): a stage hand-over of the
 * 64-vector kernels ran out.                                                 */
hlrc_status hlrc_check_device_error(hlrc_hmat M, int* code);

/* Test hook of the bounded device waits (no counterpart in the reference).
 * limit_ns > 0 replaces the 2 s bound of every device wait of the handle's
 * products (0 restores it).  skip_handover != 0 makes the next products
 * leave one hand-over undone in every CTA that waits: an H^2 tree sweep
 * announces 16 bytes more on its first level's barrier than its copies
 * deliver, and the producers of the 64-vector kernels never signal their
 * first stage.  The waiting kernel then gives up after the bound, records
 * the error bit, finishes its copies and MMAs, frees its tensor memory and
 * returns; the product is incomplete and hlrc_check_device_error reports
 * it, and the context stays usable.  Not for use during captures.           */
hlrc_status hlrc_debug_waits(hlrc_hmat M, int64_t limit_ns, int skip_handover);

/* ----------------------------------------------------- host construction
 * HLR builds its matrices with HLIBpro's clustering (TBSPCTBuilder,
 * TCardBSPPartStrat), standard admissibility (TStdGeomAdmCond), ACA
 * (approx/aca.hh:118-436) and SVD recompression (approx/svd.hh:94-197).
 * HLIBpro is closed/absent, so these are restated here on the host in C++.  */

typedef enum hlrc_problem_kind {
    HLRC_PROBLEM_LOG1D       = 0,  /* A_ij = log|x_i-x_j|, A_ii = h(log h - 1), x_i ~ U[0,1]   */
    HLRC_PROBLEM_EXP3D       = 1,  /* A_ij = exp(-|x_i-x_j|/ell) (+ nugget on diagonal), U[0,1]^3 */
    HLRC_PROBLEM_LAPLACE_SPH = 2   /* collocation 1/(4 pi r) * area_j on a refined octahedron sphere */
} hlrc_problem_kind;

typedef struct hlrc_problem {
    int32_t  kind;         /* hlrc_problem_kind                                   */
    int32_t  leaf_size;    /* cluster tree leaf size (ntile), e.g. 64             */
    int64_t  n;            /* number of points (ignored for LAPLACE_SPH)          */
    int32_t  refine;       /* LAPLACE_SPH: octahedron refinement level            */
    int32_t  uniform;      /* 1: build uniform-H (shared bases) instead of H      */
    uint64_t seed;         /* point generator seed (std::mt19937_64)              */
    double   eta;          /* admissibility parameter (2)                         */
    double   eps;          /* relative ACA/SVD accuracy (1e-6)                    */
    double   ell;          /* EXP3D correlation length                            */
    double   nugget;       /* EXP3D diagonal nugget                               */
    int32_t  nthreads;     /* host threads for the build (0 = all)                */
    int32_t  nested;       /* 1: also build the H^2 form (nested cluster bases)   */
    int32_t  on_device;    /* 1: assemble the leaves on the current CUDA device
                              (dense evaluation, ACA, QR + SVD recompression);
                              H only (not with uniform or nested); the leaf data
                              stays in device memory (hlrc_build_h_desc then
                              returns device pointers, see hlrc_build_fetch)   */
    int32_t  reserved[3];
} hlrc_problem;

typedef struct hlrc_hbuild_s* hlrc_hbuild;

hlrc_status hlrc_build(const hlrc_problem* prob, hlrc_hbuild* out);
/* descriptors pointing into the build's host storage (valid until free)     */
hlrc_status hlrc_build_h_desc(hlrc_hbuild B, hlrc_h_desc* out);
hlrc_status hlrc_build_uniform_desc(hlrc_hbuild B, hlrc_uniform_desc* out);
hlrc_status hlrc_build_h2_desc(hlrc_hbuild B, hlrc_h2_desc* out);
/* coordinates in internal order: n x dim, row-major; dim returned           */
hlrc_status hlrc_build_points(hlrc_hbuild B, const double** pts, int* dim,
                              int64_t* n);
/* per-point weights (LAPLACE_SPH: triangle areas), NULL otherwise           */
hlrc_status hlrc_build_weights(hlrc_hbuild B, const double** w);
/* internal -> external permutation (perm_i2e), length n                     */
hlrc_status hlrc_build_perm(hlrc_hbuild B, const int64_t** perm_i2e);
/* on_device builds: 1 while the leaf data is in device memory (the
 * descriptor's D, U, V and sv are device pointers; upload it with
 * hlrc_options.leaves_on_device = 1), 0 once hlrc_build_fetch copied it to
 * the host (and for host builds)                                           */
hlrc_status hlrc_build_leaves_on_device(hlrc_hbuild B, int* on_device);
/* copies device-resident leaf data to host storage and points the
 * descriptor at it (a no-op for host builds); the device copy is freed     */
hlrc_status hlrc_build_fetch(hlrc_hbuild B);
/* build statistics: seconds, number of leaves, max rank, stored bytes       */
hlrc_status hlrc_build_stats(hlrc_hbuild B, double* seconds, int64_t* nleaves,
                             int32_t* max_rank, int64_t* bytes);
hlrc_status hlrc_build_free(hlrc_hbuild B);

/* kernel entry (i,j) of the problem in internal order — used to form dense
 * reference products and to assemble leaves                                 */
double      hlrc_build_entry(hlrc_hbuild B, int64_t i, int64_t j);

#ifdef __cplusplus
}
#endif

#endif /* HLRC_H */
