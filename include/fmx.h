/*
 * fmx.h -- C ABI of the B200 FlashMatrix SpMM library (libfmx.so).
 *
 * Plain C types only: pointers, sizes, integer codes.  Device pointers are
 * CUDA device addresses on the matrix's device; `stream` is a cudaStream_t
 * passed as void* (NULL = the legacy default stream).
 *
 * Every function returns 0 (FMX_OK) or a negative fmx_status.  The text of
 * the last failure on the calling thread is returned by fmx_last_error().
 *
 * Reference interfaces replaced (paths relative to the FlashX tree):
 *   matrix/sparse_matrix_format.h:441-532   SpM_2d_index / SpM_2d_storage
 *   matrix/sparse_matrix.h:522-539,679-707  sparse_matrix::create
 *   matrix/sparse_matrix.h:629-650          sparse_matrix::multiply
 *   matrix/fm_utils.cpp:617-841             create_2d_matrix (format builder)
 */
#ifndef FMX_H
#define FMX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum fmx_status {
	FMX_OK = 0,
	FMX_ERR_INVAL = -1,      /* null pointer, bad flag, bad argument          */
	FMX_ERR_DIM = -2,        /* incompatible dimensions (sparse_matrix.cpp:712-718) */
	FMX_ERR_TYPE = -3,       /* unsupported or mismatched types (:754-766)    */
	FMX_ERR_IMAGE = -4,      /* malformed .mat / .mat_idx image               */
	FMX_ERR_OOM = -5,        /* host or device allocation failed              */
	FMX_ERR_CUDA = -6,       /* a CUDA runtime call failed                    */
	FMX_ERR_IO = -7,         /* file could not be opened / read / written     */
	FMX_ERR_UNSUPPORTED = -8 /* valid request the library does not implement  */
};

/* ---- element types ----------------------------------------------------- */
/* Dense operand types.  The numbering is this library's own. */
enum fmx_dtype {
	FMX_F32 = 0,
	FMX_F64 = 1,
	FMX_BF16 = 2, /* input only; accumulates and writes FP32 or BF16 */
	FMX_I32 = 3,
	FMX_I64 = 4
};

/* Sparse entry types stored in the image header (matrix/generic_type.h:57-70
 * prim_type order: P_BOOL=0 .. P_FLOAT=8, P_DOUBLE=9). */
enum fmx_prim_type {
	FMX_P_BOOL = 0,
	FMX_P_INTEGER = 4,
	FMX_P_LONG = 6,
	FMX_P_FLOAT = 8,
	FMX_P_DOUBLE = 9
};

typedef struct fmx_matrix fmx_matrix; /* a matrix resident on one GPU */
typedef struct fmx_image fmx_image;   /* a host-side .mat/.mat_idx pair  */

const char *fmx_strerror(int status);
const char *fmx_last_error(void);
/* Library version string, e.g. "fmx 0.1 sm_100a". */
const char *fmx_version(void);

/* ---- matrix images (host) ------------------------------------------------
 * A matrix image is the reference's on-disk 2D format: a 4096-byte
 * matrix_header page followed by block rows of packed sparse_block_2d tiles
 * (.mat), plus an index of header + (nbrows+1) int64 byte offsets (.mat_idx).
 * Replaces SpM_2d_index::load / SpM_2d_storage::load
 * (matrix/sparse_matrix_format.cpp:238-306) and ::dump (:164-181,417-420).
 */

/* Builder flags (matrix/fm_utils.cpp:37-49, 444-482). */
#define FMX_BUILD_DEDUP 0x1          /* set_deduplicate(true)                  */
#define FMX_BUILD_KEEP_SELF_LOOPS 0x2 /* set_remove_self_edge(false)            */
#define FMX_BUILD_REF_VALUE_LAYOUT 0x4 /* place tile values the way the reference
                                         builder does (fm_utils.cpp:240-241,259-260
                                         copy each tile's values from the start of
                                         the row); default keeps each entry's own value */

/* Build an image from an edge list (src[i] -> dst[i], optional values of
 * `val_type` (FMX_P_BOOL = no values, FMX_P_FLOAT, FMX_P_DOUBLE, FMX_P_INTEGER,
 * FMX_P_LONG)).  nrows/ncols = 0 means max id + 1 (fm_utils.cpp:730-739,788).
 * block_h/block_w: powers of two <= 32768 (matrix_header.h:42-62).
 * Replaces fm::create_2d_matrix (matrix/fm_utils.cpp:617-715,726-841). */
int fmx_image_build(const uint32_t *src, const uint32_t *dst, const void *vals,
                    int val_type, uint64_t nedges, uint64_t nrows, uint64_t ncols,
                    uint32_t block_h, uint32_t block_w, int flags, int nthreads,
                    fmx_image **out);
/* Wrap copies of an existing .mat_idx / .mat byte pair (validated). */
int fmx_image_from_bytes(const void *idx, size_t idx_len, const void *mat,
                         size_t mat_len, fmx_image **out);
int fmx_image_load(const char *mat_idx_path, const char *mat_path, fmx_image **out);
int fmx_image_dump(const fmx_image *img, const char *mat_idx_path, const char *mat_path);
/* Borrow the bytes of an image (valid until fmx_image_free). */
int fmx_image_bytes(const fmx_image *img, const void **idx, size_t *idx_len,
                    const void **mat, size_t *mat_len);
/* nrows, ncols, nnz, entry size in bytes (0 = binary), prim type, block h, w. */
int fmx_image_info(const fmx_image *img, uint64_t *nrows, uint64_t *ncols,
                   uint64_t *nnz, uint32_t *entry_size, int *prim_type,
                   uint32_t *block_h, uint32_t *block_w);
/* Check every tile invariant (sparse_matrix_format.cpp:36-60,371-415). */
int fmx_image_verify(const fmx_image *img);
int fmx_image_free(fmx_image *img);

/* ---- GPU-resident matrices ------------------------------------------------
 * Replaces sparse_matrix::create(SpM_2d_index::ptr, SpM_2d_storage::ptr[,
 * t_index, t_storage]) (matrix/sparse_matrix.cpp:679-707).  The image is
 * decoded on the host and its tiles are kept resident in HBM of `device`
 * with int32 column indices.  `t_img` (nullable) is the transpose image of an
 * asymmetric matrix (block_sparse_asym_matrix, sparse_matrix.cpp:582-665).
 */
int fmx_matrix_create(const fmx_image *img, const fmx_image *t_img, int device,
                      fmx_matrix **out);
/* The semi-external form: sparse_matrix::create(SpM_2d_index::ptr,
 * safs::file_io_factory::shared_ptr[, t_index, t_mat_io_fac])
 * (matrix/sparse_matrix.cpp:693-707) keeps the tiles in SAFS and reads them
 * during every multiply.  Here the matrix's entry stream (column ids and
 * values) stays in pinned host memory and every SpMM streams it to the GPU in
 * slices of about slice_entries entries (0: 2^26), copying one slice while
 * the kernel runs on the previous one; the schedule, the hot-column pack and
 * the partial sums stay in HBM.  For matrices whose entry stream does not fit
 * in HBM beside the dense operands.  Results are identical to
 * fmx_matrix_create's. */
int fmx_matrix_create_streamed(const fmx_image *img, const fmx_image *t_img, int device,
                               uint64_t slice_entries, fmx_matrix **out);
/* Slices per SpMM (0 for a resident matrix) and pinned host bytes held. */
int fmx_matrix_stream_info(const fmx_matrix *m, uint64_t *slices, uint64_t *host_bytes);
/* Build the resident matrix straight from an edge list in the memory of
 * `device` (src_dev, dst_dev: uint32 ids; vals_dev: nedges values of
 * val_type, or NULL for FMX_P_BOOL): the sort, deduplication and row
 * pointers of fm::create_2d_matrix (matrix/fm_utils.cpp:267-433) run on the
 * GPU, the work schedule on the host, with no .mat image in between.  The
 * same entries in the same order as fmx_image_build + fmx_matrix_create with
 * the same flags, so SpMM results are identical.  flags: FMX_BUILD_DEDUP,
 * FMX_BUILD_KEEP_SELF_LOOPS, FMX_BUILD_TRANSPOSE (also build A^T, the
 * asymmetric pair create_2d_matrix makes for a directed graph).  nrows /
 * ncols = 0: the largest id + 1.  Fewer than 2^31 edges.  Synchronises
 * `stream`. */
#define FMX_BUILD_TRANSPOSE 0x8
int fmx_matrix_build_device(const uint32_t *src_dev, const uint32_t *dst_dev,
                            const void *vals_dev, int val_type, uint64_t nedges,
                            uint64_t nrows, uint64_t ncols, int flags, int device,
                            void *stream, fmx_matrix **out);
/* Convenience: fmx_image_load + fmx_matrix_create (+ free of the images). */
int fmx_matrix_load(const char *mat_idx_path, const char *mat_path,
                    const char *t_mat_idx_path, const char *t_mat_path,
                    int device, fmx_matrix **out);
/* The FlashGraph 1D format: fg::create_sparse_matrix(FG_graph::ptr,
 * entry_type) (flash-graph/fg_sparse_matrix.cpp:577-590) over a graph image
 * (the adjacency file FG_graph::create reads: graph_header page, then one
 * ext_mem_undirected_vertex record per vertex, flash-graph/vertex.h:444-562;
 * a directed graph's in-edge records, then its out-edge records).  Row i is
 * vertex i's out-edge list (A), its in-edge list for the transpose; an
 * undirected graph gives a symmetric matrix.  Every stored neighbor counts,
 * in record order (duplicates and self-loops included), which is the order
 * fg_row_spmm_task::run_on_row sums in (fg_sparse_matrix.cpp:83-106).
 * val_type: FMX_P_BOOL for a graph without edge data, else the edge data's
 * type, whose size must equal the header's edge_data_size (the reference's
 * assertion, :476-478,551-553).  The vertex index file is not needed: the
 * records are walked in order.  Time-series graphs: FMX_ERR_UNSUPPORTED. */
int fmx_matrix_from_fg(const void *adj, size_t adj_len, int val_type, int device,
                       fmx_matrix **out);
int fmx_matrix_load_fg(const char *adj_path, int val_type, int device, fmx_matrix **out);
int fmx_matrix_info(const fmx_matrix *m, uint64_t *nrows, uint64_t *ncols,
                    uint64_t *nnz, int *prim_type, int *symmetric);
/* Device bytes held by the matrix (tiles, schedule, scratch). */
int fmx_matrix_device_bytes(const fmx_matrix *m, uint64_t *bytes);
/* sparse_matrix::transpose (sparse_matrix.cpp:514-516,619-626): a symmetric
 * matrix returns itself; an asymmetric pair swaps its two images.  The
 * returned handle shares device memory with `m` and must be freed with
 * fmx_matrix_free before or after `m`. */
int fmx_matrix_transpose(const fmx_matrix *m, fmx_matrix **out);
int fmx_matrix_free(fmx_matrix *m);

/* The solvers (fmx_eigen_solve, fmx_pagerank, the GNN, the device builder)
 * take their device workspace from one memory pool per device that keeps
 * freed memory reserved for the next call.  Hand it back to the driver (as
 * torch.cuda.empty_cache does for torch's cache). */
int fmx_release_cached(int device);

/* ---- SpMM -----------------------------------------------------------------
 * Y = diag(row_scale_out) * A * diag(row_scale_in) * X   (scales nullable)
 * Replaces sparse_matrix::multiply(in, out) (matrix/sparse_matrix.cpp:709-771)
 * and the spmm_creator<DenseType, SparseType> tasks (sparse_matrix.h:219-436).
 *   X: ncols x k, row-major, leading dimension ldx (elements), type x_type
 *   Y: nrows x k, row-major, leading dimension ldy, type y_type; fully
 *      overwritten (block_spmm_task::notify_complete, sparse_matrix.cpp:354-393)
 *   Supported (x_type -> y_type): F32->F32, F64->F64, BF16->F32, BF16->BF16,
 *   I32->I32, I64->I64.  A binary matrix multiplies by 1; a weighted matrix's
 *   entries are converted to the accumulation type (float entries with F64
 *   operands reproduce spmm_creator<double,float>, test-eigen.cpp:47).
 *   Scales have the accumulation type (float for F32/BF16, double for F64).
 * Each output row is summed in ascending column order by one lane group, the
 * reference's order, except rows longer than the split threshold, which are
 * summed as fixed-order partial chunks.  Asynchronous on `stream`. */
/* Rows with at most this many entries are summed by one lane group in the
 * reference's order; their results are bit-identical to the reference's. */
#define FMX_EXACT_ROW_MAX 256

int fmx_spmm(const fmx_matrix *m, int x_type, const void *X, int64_t ldx,
             int y_type, void *Y, int64_t ldy, int64_t k,
             const void *row_scale_in, const void *row_scale_out, void *stream);

/* FP32 SpMM that allocates nothing (no counterpart in the reference).
 * For callers that must not allocate device memory while they run: code
 * inside a memory pool or arena that owns the device's memory, allocator
 * callbacks, real-time or signal-driven paths.  Same arguments and results as
 * fmx_spmm with x_type = y_type = FMX_F32 and no row scales, for binary or
 * float-weighted matrices.  Its scratch is one fixed 32 MiB array compiled
 * into libfmx, present on every GPU that loads the library until the process
 * exits.  A matrix needs H + 1024 * P bytes of it, where H is
 * (n_hot_cols + 1) * 128 rounded up to a multiple of 256 and P the number of
 * chunk-sum slots (from fmx_matrix_hot: P = (scratch_bytes - (n_hot_cols + 1)
 * * 128) / 2048); matrices that need more than 32 MiB are rejected with
 * FMX_ERR_UNSUPPORTED.  The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress) and keeps it for the life of the
 * process, so make that first call before any stream capture; a device reset
 * (cudaDeviceReset) while the library is loaded is not supported by this
 * entry point.  All calls share the array: calls that overlap on the GPU (on
 * different streams, or from different threads) race and must not be
 * issued. */
int fmx_spmm_noalloc(const fmx_matrix *m, const float *X, int64_t ldx, float *Y,
                     int64_t ldy, int64_t k, void *stream);

/* Host-buffer SpMM: copies X in and Y out through the device (pinned or
 * pageable host memory), synchronous.  The e2e path a CPU caller uses. */
int fmx_spmm_host(const fmx_matrix *m, int x_type, const void *X_host, int64_t ldx,
                  int y_type, void *Y_host, int64_t ldy, int64_t k);

/* Host-buffer SpMM, asynchronous (no counterpart in the reference, whose
 * multiply is synchronous): enqueues the copy of X to the device, the SpMM
 * and the copy of Y back, and returns.  The call ends on `stream` when Y has
 * arrived: X_host and Y_host must stay valid until then (synchronise the
 * stream or wait on an event recorded after the call).  With pinned host
 * memory (cudaHostAlloc, cudaHostRegister) the copies are asynchronous;
 * pageable memory makes them synchronous.  The matrix keeps two device
 * staging slots (grow-only, freed with the matrix) and two streams of its
 * own: the copies of X run back to back on one and the copies of Y on the
 * other, while each SpMM runs on `stream`, so calls issued alternately on two
 * streams overlap one call's copy of Y with the next call's copy of X (PCIe
 * carries both directions at once).  The SpMMs of these calls run one after
 * another, ordered by an event, because they share the matrix's scratch;
 * they are not ordered against fmx_spmm calls on other streams.  Calls on
 * one matrix from several host threads are serialised by a lock, but their
 * stream order is the caller's to set. */
int fmx_spmm_host_async(const fmx_matrix *m, int x_type, const void *X_host, int64_t ldx,
                        int y_type, void *Y_host, int64_t ldy, int64_t k, void *stream);

/* Work decomposition of the resident matrix: rows summed by one lane group,
 * work ranges (runs of whole rows, or chunks of rows longer than
 * FMX_EXACT_ROW_MAX), rows finished by the chunk-sum pass, and kernel
 * launches per 128-byte column panel of one fmx_spmm. */
int fmx_matrix_schedule(const fmx_matrix *m, uint64_t *n_light_rows, uint64_t *n_split_tasks,
                        uint64_t *n_heavy_rows, uint64_t *kernels_per_spmm);

/* Hot-column pack of the resident matrix: columns whose X rows each SpMM
 * packs into scratch (the highest in-degrees, up to 2^20), the entries that
 * read the pack, and the scratch bytes held (pack + long-row partial sums). */
int fmx_matrix_hot(const fmx_matrix *m, uint64_t *n_hot_cols, uint64_t *hot_entries,
                   uint64_t *scratch_bytes);

/* A 64-bit FNV-1a digest of one resident orientation (transpose = 0: A,
 * else A^T): the entry stream, values, ranges, heavy-row list, hot columns
 * and the schedule counts.  Two builds of the same matrix (a host image
 * through fmx_matrix_create, device edges through fmx_matrix_build_device)
 * lay it out identically exactly when the digests agree.  Copies the layout
 * to the host: a diagnostic, not for hot paths.  No reference counterpart. */
int fmx_matrix_layout_digest(const fmx_matrix *m, int transpose, uint64_t *digest);

/* ---- dense kernels of the block eigensolver --------------------------------
 * Tall-skinny products over n-row, row-major FP32 blocks of at most 64
 * columns (block_multi_vector::gemm / MvTransMv / MvNorm,
 * matrix/eigensolver/block_dense_matrix.cpp:997-1530).  Precision:
 *   FMX_DENSE_BF16    tensor cores (tcgen05), BF16 operands, FP32 accumulate
 *   FMX_DENSE_TF32X3  tensor cores, each operand split x = hi + lo in TF32 and
 *                     hi*hi + hi*lo + lo*hi accumulated in FP32 (FP32 accuracy)
 *   FMX_DENSE_F64     CUDA cores, FP64 accumulate (Gram only)
 * `err` (device int) is set to 1 if a tensor-core wait ran out of time. */
#define FMX_DENSE_BF16 0
#define FMX_DENSE_TF32X3 1
#define FMX_DENSE_F64 2

/* Y (n x N) = X (n x K) * B (K x N); K, N <= 64; B row-major (ldb). */
int fmx_dense_gemm(int precision, const float *X, int64_t ldx, int64_t n, int K,
                   const float *B, int ldb, int N, float *Y, int64_t ldy, int *err,
                   void *stream);
/* Number of per-CTA partials the Gram of n rows uses (size of `part`:
 * parts * M * N elements of float, or double for FMX_DENSE_F64). */
int fmx_dense_gram_parts(int precision, int64_t n);
/* G (M x N, row-major) = X^T W over n rows; float G, or double for F64.
 * Partials are added in a fixed order (deterministic). */
int fmx_dense_gram(int precision, const float *X, int64_t ldx, int M, const float *W,
                   int64_t ldw, int N, int64_t n, void *part, void *G, int *err,
                   void *stream);
/* T = R^-1 where G = R^T R (upper Cholesky), FP64, b <= 64; *info = 0 or
 * the 1-based column of the first non-positive pivot. */
int fmx_dense_chol_inv(const double *G, int b, double *T, int *info, void *stream);
/* H = V diag(w) V^T (symmetric, FP64, b <= 64), eigenvalues descending. */
int fmx_dense_sym_eig(const double *H, int b, double *w, double *V, void *stream);

/* ---- block eigensolver -------------------------------------------------------
 * Largest eigenpairs of the symmetric operator diag(s) A diag(s) (s = NULL:
 * A itself) by Chebyshev-filtered subspace iteration on a block of
 * block_size vectors.  Replaces fm::eigen::compute_eigen
 * (matrix/eigensolver/eigensolver.h:74-75, eigensolver.cpp:118-308); the
 * option and status fields mirror eigen_options (eigensolver.h:59-73) and
 * eigen_res::eigen_status (:51-54). */
#define FMX_EIGEN_LA 0      /* largest algebraic ("LA") */
#define FMX_EIGEN_LM 1      /* largest magnitude ("LM", the reference's default) */
#define FMX_EIGEN_OP_SCALED 0
#define FMX_EIGEN_OP_GRAM 1
#define FMX_EIGEN_PLAIN 0   /* FP32 SpMM operands; dense products in FP64 on CUDA cores */
#define FMX_EIGEN_MIXED 1   /* filter in correction form with BF16 SpMM operands (FP32
                               accumulation), Rayleigh-Ritz SpMM in FP32; CholQR basis
                               update on tensor cores (3xTF32) until tensor_until, FP64
                               after; Gram products, Cholesky, projected problem and
                               residual norms in FP64 */

typedef struct fmx_eigen_options {
	int nev;            /* wanted eigenpairs (eigen_options::nev) */
	int block_size;     /* vectors per block, nev <= block_size <= 64 */
	int degree;         /* largest Chebyshev degree of a filter pass (SpMMs per pass);
	                       each pass picks the degree its slowest wanted residual needs */
	int max_iters;      /* filter passes (eigen_options::max_iters) */
	int which;          /* FMX_EIGEN_LA or FMX_EIGEN_LM (eigen_options::which) */
	int precision;      /* FMX_EIGEN_PLAIN or FMX_EIGEN_MIXED */
	double tol;         /* residual ||A x - l x|| / ||A|| every wanted pair must meet */
	double lower;       /* lower bound of the spectrum (-1 for D^-1/2 A D^-1/2) */
	double upper;       /* upper bound of the spectrum (1 for D^-1/2 A D^-1/2); ||A|| is
	                       taken as max(|lower|, |upper|) */
	double tensor_until;/* FMX_EIGEN_MIXED: dense products on tensor cores while the
	                       largest residual exceeds this */
	uint64_t seed;      /* random start block, uniform(-1, 1) (MvRandom) */
	const float *X0;    /* optional start block on the device (n x block_size), or NULL */
	int64_t ldx0;
	int op;             /* FMX_EIGEN_OP_SCALED: diag(s) A diag(s) (A square);
	                       FMX_EIGEN_OP_GRAM: A^T A on ncols-vectors, through the
	                       transpose (SVD_Operator, matrix/test/test-eigen.cpp:138-177):
	                       its eigenpairs are the squared singular values and right
	                       singular vectors of A; the bounds must enclose
	                       [0, sigma_max^2] and no row scale is taken */
} fmx_eigen_options;

typedef struct fmx_eigen_status {
	int iters;          /* filter passes (eigen_status::num_iters) */
	int converged;      /* wanted pairs whose explicit residual meets tol */
	int64_t num_ops;    /* SpMM columns applied (eigen_status::num_ops) */
	int64_t spmm_calls;
	double max_residual;/* largest explicit residual of the wanted pairs */
	double seconds;     /* wall time of the call */
} fmx_eigen_status;

/* Defaults as eigen_options() and init(nev) (eigensolver.cpp:82-116): tol 1e-8,
 * max_iters 500, block_size max(2 nev, 16) (at most 64), degree 16, LA, plain,
 * spectrum [-1, 1], seed 1, op FMX_EIGEN_OP_SCALED. */
void fmx_eigen_default_options(fmx_eigen_options *opts, int nev);

/* Solve; evals and residuals are host arrays of nev, evecs a device array of
 * n x nev (row-major, ldv), any of them NULL when not wanted.  The residuals
 * are those of the returned vectors, from an explicit final product.  A run
 * that stops at max_iters returns FMX_OK with status->converged < nev. */
int fmx_eigen_solve(const fmx_matrix *m, const float *row_scale,
                    const fmx_eigen_options *opts, double *evals, float *evecs,
                    int64_t ldv, double *residuals, fmx_eigen_status *status,
                    void *stream);

/* s = D^-1/2 with D = A 1 (row sums; 0 where a row is empty), the scaling of
 * NA_eigen_Operator (matrix/test/test-eigen.cpp:96-109); s is a device array
 * of n floats. */
int fmx_na_scale(const fmx_matrix *m, float *s, void *stream);

/* ---- PageRank ------------------------------------------------------------------
 * fm::alg::PageRank(mat, max_niters, damping, num_in_mem)
 * (matrix/libmatrix-algs/PageRank.cpp:63-133) with the reference's float
 * arithmetic: out-degrees A 1 clamped to >= 1, pr = 1/n, then while fewer than
 * n vertices changed by less than 0.001/n and fewer than max_iters iterations
 * ran: in = pr / deg, out = A^T in, pr = out * damping + (1 - damping) / n.
 * `m` needs its transpose (an asymmetric matrix created with t_img, or a
 * symmetric one).  pr: n device floats (the result); *iters: iterations run.
 * Synchronises the stream once per iteration (the convergence test). */
int fmx_pagerank(const fmx_matrix *m, uint64_t max_iters, float damping, float *pr,
                 uint64_t *iters, void *stream);

/* ---- learned warm start ---------------------------------------------------------
 * A 2-layer graph network that maps vertex features to a start block for
 * fmx_eigen_solve (no counterpart in the reference):
 *   F  (n x 16)  standardised log(1 + degree), then 15 N(0,1) channels (seeded)
 *   Z  (n x 64)  [F, A_s F, A_s^2 F, A_s^3 F]    (A_s = diag(s) A diag(s))
 *   H  (n x 64)  relu(Z W1 + b1)
 *   Y  (n x 16)  A_s (H W2)
 * trained to align span(Y) with given eigenvectors U (loss 1 - ||U^T Q||_F^2 /
 * nev, Q an orthonormal basis of span(Y)).  Weights are FP32 master copies
 * (Adam) that enter every product as BF16 (FMX_DENSE_BF16: tcgen05, FP32
 * accumulation) or split 3xTF32 (FMX_DENSE_TF32X3, for gradient checks).
 * Parameters, flat: W1 (64 x 64, row-major), b1 (64), W2 (64 x 16). */
#define FMX_GNN_FEATURES 64
#define FMX_GNN_OUT 16
#define FMX_GNN_PARAMS 5184

typedef struct fmx_gnn fmx_gnn;
/* Glorot-uniform weights from `seed`, zero bias, zero optimiser state. */
int fmx_gnn_create(int device, uint64_t seed, fmx_gnn **out);
int fmx_gnn_free(fmx_gnn *g);
/* Copy FMX_GNN_PARAMS floats in (resets the optimiser state) or out. */
int fmx_gnn_set_params(fmx_gnn *g, const float *host);
int fmx_gnn_get_params(const fmx_gnn *g, float *host);
/* Z (n x 64 device floats, 16-byte aligned) for matrix m and its
 * D^-1/2 row scale (fmx_na_scale; required: the degree feature is read
 * back from it as 1 / s^2). */
int fmx_gnn_features(const fmx_matrix *m, const float *row_scale, uint64_t seed,
                     float *Z, void *stream);
/* Y (n x 16 device floats). */
int fmx_gnn_forward(const fmx_gnn *g, const fmx_matrix *m, const float *row_scale,
                    const float *Z, int precision, float *Y, void *stream);
/* Forward, loss against U (n x nev device floats, ldu), backward into the
 * model's gradient buffer; *loss (host) and grad_host (FMX_GNN_PARAMS floats)
 * are optional.  Synchronises the stream. */
int fmx_gnn_loss_grad(fmx_gnn *g, const fmx_matrix *m, const float *row_scale,
                      const float *Z, const float *U, int64_t ldu, int nev,
                      int precision, double *loss, float *grad_host, void *stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) with the stored gradient. */
int fmx_gnn_adam_step(fmx_gnn *g, float lr, void *stream);

/* ---- synthetic graphs ---------------------------------------------------------
 * R-MAT edges (a,b,c; d = 1-a-b-c) of 2^scale vertices, counter-based so the
 * host and device streams are identical.  `permute` relabels vertices by a
 * seeded bijection (Boost rmat_iterator permute_vertices, used by
 * flash-graph/tools/rmat-gen.cpp:43-44). */
int fmx_rmat_edges_host(int scale, uint64_t nedges, double a, double b, double c,
                        uint64_t seed, int permute, uint32_t *src, uint32_t *dst,
                        int nthreads);
int fmx_rmat_edges_device(int scale, uint64_t nedges, double a, double b, double c,
                          uint64_t seed, int permute, uint32_t *src_dev,
                          uint32_t *dst_dev, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* FMX_H */
