/*
 * flagsparse_b200.h -- C ABI of the B200 (sm_100a) sparse-matrix kernels.
 *
 * Every entry point takes plain device pointers, element counts and a CUDA
 * stream handle (cudaStream_t passed as void*), enqueues its kernels on that
 * stream and returns a status code.  No entry point allocates device memory,
 * synchronises the stream or reads device data on the host: scratch memory is
 * passed in by the caller (its size comes from fsb_workspace_bytes).
 *
 * The Python package flagsparse_public_b200 binds these through ctypes and
 * keeps the FlagSparse operator API (prepare_* / flagsparse_* functions) on
 * top.  Each declaration names the FlagSparse launch it replaces; paths are
 * relative to the FlagSparse project root.
 */
#ifndef FLAGSPARSE_B200_H
#define FLAGSPARSE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FSB_ABI_VERSION 2

/* ---- status codes ------------------------------------------------------ */
#define FSB_OK               0
#define FSB_ERR_INVALID     -1  /* bad argument (null pointer, bad size, bad plan) */
#define FSB_ERR_UNSUPPORTED -2  /* dtype / mode combination not compiled in       */
#define FSB_ERR_LAUNCH      -3  /* cudaGetLastError() reported a launch failure    */
#define FSB_ERR_WORKSPACE   -4  /* workspace missing or smaller than required      */
#define FSB_ERR_TIMEOUT     -5  /* a bounded device wait gave up                   */
#define FSB_ERR_LIMIT       -6  /* size exceeds a fixed limit of the entry point   */

/* ---- element type codes ------------------------------------------------ */
#define FSB_F16   0
#define FSB_BF16  1
#define FSB_F32   2
#define FSB_F64   3
#define FSB_C64   4   /* interleaved (re, im) float pairs  */
#define FSB_C128  5   /* interleaved (re, im) double pairs */
#define FSB_I32   6
#define FSB_I64   7
#define FSB_C32   8   /* interleaved (re, im) float16 pairs (torch complex32),
                         accumulated in float32 pairs                       */

/* ---- accumulation modes ------------------------------------------------
 * NATIVE : f16/bf16 -> f32, f32 -> f32, f64 -> f64, c64 -> f32 pairs
 *          (the FlagSparse "opt" paths: spmv_csr.py:246, spmm_csr.py:631)
 * WIDE   : f16/bf16 -> f32, f32 -> f64, c64 -> f64 pairs, f64 -> f64
 *          (the FlagSparse plain paths: spmv_csr.py:116-121,
 *           spmm_csr.py:544-551, spmm_coo.py:11-18)
 * COMP   : f16/bf16/f32 values, f32 accumulation with error-free
 *          transformations (TwoProduct by FMA + TwoSum, Ogita-Rump-Oishi
 *          Dot2) on rows longer than plan->comp_threshold nonzeros.      */
#define FSB_ACC_NATIVE 0
#define FSB_ACC_WIDE   1
#define FSB_ACC_COMP   2

/* ---- algorithms ------------------------------------------------------- */
#define FSB_ALGO_ROWS   0  /* one group of plan->lanes lanes per row        */
#define FSB_ALGO_MERGE  1  /* merge-path units over (rows + nonzeros)      */
#define FSB_ALGO_FLAT   2  /* SpMM: merge-path units, one warp streams the
                              unit's nonzeros, B rows gathered to registers */
#define FSB_ALGO_GATHER 3  /* SpMM: merge-path units, B rows gathered into a
                              shared-memory ring by TMA bulk copies
                              (cp.async.bulk + mbarrier), several stages deep */
#define FSB_ALGO_SEQ    4  /* SpMM: merge-path units, the warp walks a unit's
                              nonzeros in batches of up to 32 (32 / LPN per
                              step, 16-byte lane vectors over a column tile),
                              B rows gathered to registers, rows reduced
                              across sub-groups only at row ends            */

/* ---- plan flags (fsb_plan.flags) ------------------------------------- */
#define FSB_PLAN_TMA_GATHER 1  /* SEQ: B rows staged in a per-warp shared-memory
                                  ring by TMA row gathers (tile::gather4, four
                                  B rows per instruction), several stages ahead
                                  of the multiply-adds; float32 / float16 /
                                  bfloat16 values, float accumulators, 16-byte
                                  aligned B and C rows, else
                                  FSB_ERR_UNSUPPORTED                          */

#define FSB_PLAN_OVERLAP_LAUNCH 2  /* ROWS SpMV of at most 592 CTAs: launched
                                  with programmatic dependent launch, so its
                                  CTAs may start while the previous kernel on
                                  the stream drains; each waits for that
                                  kernel's completion (griddepcontrol.wait)
                                  before reading anything, and lets the next
                                  such launch start early.  Hides the launch
                                  gap of back-to-back SpMVs (solver loops,
                                  CUDA graphs); results are unchanged       */

/* A CSR matrix (or a sorted COO matrix seen as row runs).
 * row_ptr has n_rows + 1 entries.  If row_map is non-null, row r of this
 * structure is written to output row row_map[row_ptr[r]] (COO row runs:
 * row_ptr = seg_starts, row_map = the sorted COO row array).              */
typedef struct fsb_csr {
    const void* values;
    const void* col_idx;
    const void* row_ptr;
    const void* row_map;
    int32_t value_dtype;    /* FSB_F16 .. FSB_C128, FSB_C32 */
    int32_t index_dtype;    /* FSB_I32 / FSB_I64, col_idx */
    int32_t ptr_dtype;      /* FSB_I32 / FSB_I64, row_ptr */
    int32_t row_map_dtype;  /* FSB_I32 / FSB_I64, row_map */
    int64_t n_rows;
    int64_t n_cols;
    int64_t nnz;
} fsb_csr;

/* Launch plan chosen by the host (heuristic, autotuner or learned selector). */
typedef struct fsb_plan {
    int32_t algo;            /* FSB_ALGO_ROWS / FSB_ALGO_MERGE                     */
    int32_t lanes;           /* ROWS: lanes per row group, power of two in [1, 32] */
    int32_t items_per_unit;  /* merge-path plans: items (rows + nnz) per unit,
                                1 .. 2^24 for SpMM                               */
    int32_t n_tile;          /* SpMM: dense columns per column tile, 0 = all       */
    int64_t n_units;         /* MERGE: number of units                             */
    const int64_t* unit_coords; /* MERGE: device array [(n_units + 1) * 2] of
                                   (row, nnz) unit start coordinates              */
    int64_t row_cap;         /* > 0: nonzeros consumed per row are capped
                                (FlagSparse max_segments * block_nnz)             */
    int64_t comp_threshold;  /* FSB_ACC_COMP: rows longer than this are
                                compensated (FlagSparse precision form: 4096)     */
    int32_t grid_blocks;     /* ROWS, SEQ: CTAs to launch (SEQ: a persistent grid
                                striding over the units), 0 = automatic           */
    int32_t flags;           /* FSB_PLAN_* bits, 0 = none                          */
    /* SEQ only, optional (null: split rows finish in a second kernel).
     * unit_runs [n_units * 2] from fsb_merge_runs for the same unit_coords;
     * tickets: ticket_slots int32 counters, zero-filled by the caller once
     * when allocated, at least n_units * (column tiles of the call) of them.
     * With both, the kernel finishes each split row itself: every unit that
     * holds part of the row stores its partial, then takes a ticket; the unit
     * drawing the last ticket adds the row's partials in unit order (the same
     * sums as the second kernel) and stores the row.  No unit ever waits.  The
     * counters return to zero by the end of every call; calls sharing one
     * ticket array must not overlap on the GPU.                            */
    const int64_t* unit_runs;
    int32_t* tickets;
    int64_t ticket_slots;
} fsb_plan;

int         fsb_abi_version(void);
const char* fsb_status_string(int status);
/* Text of the last error recorded by this thread (launch errors, bad plans). */
const char* fsb_last_error(void);

/* Sticky device error word of the kernels that wait on mbarriers: 0, or
 * FSB_ERR_TIMEOUT when a bounded wait gave up (the kernel then drained its
 * copies in flight and returned).  Synchronises the current device; with
 * reset != 0 the word is cleared.                                           */
int fsb_device_error(int* status_out, int reset);

/* Self-test of the bounded waits: one warp waits on an mbarrier that no
 * thread or copy ever completes; after limit_ns (at most 2 s) it gives up and
 * records FSB_ERR_TIMEOUT in the device error word, leaving the context
 * usable.  No FlagSparse counterpart (failure-path test hook).             */
int fsb_selftest_wait_timeout(int64_t limit_ns, void* stream);

/* Scratch bytes fsb_spmv_csr / fsb_spmm_csr need for this plan (0 for ROWS). */
int64_t fsb_workspace_bytes(int is_spmm, const fsb_csr* A, int64_t n_dense,
                            int acc_mode, int out_dtype, const fsb_plan* plan);

/* Merge-path partition: unit_coords[2*u], unit_coords[2*u+1] = (row, nnz)
 * coordinate of path diagonal u * items_per_unit, for u in [0, n_units], the
 * last one clamped to (n_rows, nnz).  With snap_threshold > 0 a boundary that
 * falls inside a row shorter than snap_threshold nonzeros is moved back to the
 * start of that row (fewer split rows).  n_units must be
 * ceil((n_rows + nnz) / items_per_unit).
 * Replaces the host-side long-row split of spmm_csr.py:417-441 and the
 * per-bucket torch.nonzero launches of spmv_csr.py:345-391.               */
int fsb_merge_partition(const void* row_ptr, int ptr_dtype, int64_t n_rows,
                        int64_t nnz, int32_t items_per_unit,
                        int64_t snap_threshold, int64_t* unit_coords,
                        int64_t n_units, void* stream);

/* Structural check of a CSR matrix in two kernels (per-CTA figures into
 * workspace, then one CTA folding them into out[]) in place of FlagSparse's
 * separate device reductions and host reads (spmv_csr.py:524-541,
 * spmm_csr.py:197-255).  No memset and no copy: out[] may be device memory
 * or pinned host memory (read it after synchronising the stream), so the
 * check never queues behind host<->device copies.  out: eight int64:
 *   out[0] = row_ptr[0]             out[1] = row_ptr[n_rows]
 *   out[2] = rows of negative length
 *   out[3] = column indices below zero
 *   out[4] = largest non-negative column index (0 when there is none)
 *   out[5] = longest row            out[6] = sum of squared row lengths
 *   out[7] = empty rows   (out[5..7] over the rows of non-negative length)
 * workspace_bytes >= fsb_csr_check_workspace_bytes(n_rows, nnz).         */
int64_t fsb_csr_check_workspace_bytes(int64_t n_rows, int64_t nnz);
int fsb_csr_check(const void* row_ptr, int ptr_dtype, int64_t n_rows,
                  const void* col_idx, int index_dtype, int64_t nnz,
                  int64_t* out, void* workspace, int64_t workspace_bytes,
                  void* stream);

/* Split-row runs of a merge-path partition (unit_coords from
 * fsb_merge_partition for the same row_ptr): for every unit u whose end falls
 * inside a row r (after at least one of r's nonzeros), unit_runs[2*u] is the
 * first and unit_runs[2*u+1] the last unit holding part of r (the last one
 * holds r's end); -1, -1 for the other units.  Computed once per partition
 * (binary searches over the coordinates).  Replaces the per-call host loop
 * over long rows of _build_spmm_opt_split_metadata (spmm_csr.py:417-441).  */
int fsb_merge_runs(const void* row_ptr, int ptr_dtype, int64_t n_rows,
                   const int64_t* unit_coords, int64_t n_units,
                   int64_t* unit_runs, void* stream);

/* One-shot SpMV with the structural check, for a matrix seen once (the
 * reference's flagsparse_spmv_csr without `prepared`: prepare_spmv_csr's
 * checks, spmv_csr.py:497-549, then the product, :796-872).  One host call:
 * fsb_csr_check (partials in workspace) writing its eight figures to a
 * pinned buffer of the calling thread, one stream synchronisation, the
 * figures copied to figures[] (host memory); a
 * malformed structure (row_ptr[0] != 0, row_ptr[n_rows] != nnz, a negative
 * row length, a column outside [0, n_cols)) returns FSB_ERR_INVALID with
 * nothing launched, so the caller raises its own error from the figures.
 * Otherwise the plan follows from the figures (merge path when the longest
 * row exceeds 8 x max(mean, 1) + 256 and the mean is below 32, else
 * 2 x mean / (16-byte vector elements) lanes per row group, a power of two
 * in [2, 32]), written to plan_out when non-null, and the product runs as
 * fsb_spmv_csr.  workspace_bytes >= fsb_spmv_csr_checked_workspace_bytes.  */
int64_t fsb_spmv_csr_checked_workspace_bytes(const fsb_csr* A, int acc_mode,
                                             int out_dtype);
int fsb_spmv_csr_checked(const fsb_csr* A, const void* x, void* y,
                         int out_dtype, int acc_mode, void* workspace,
                         int64_t workspace_bytes, int64_t* figures,
                         fsb_plan* plan_out, void* stream);

/* Allocation-free merge-path SpMV, y = A x, for callers that cannot allocate
 * device memory (a C program or plug-in handed device pointers by a host
 * framework that owns all device memory, or a latency-critical loop that
 * cannot afford cudaMalloc's implicit synchronisation).  No counterpart in
 * FlagSparse.  Same arguments and results as fsb_spmv_csr with a merge-path
 * plan of items_per_unit items per tile (128 x [1, 8], unsnapped), but the
 * tile coordinates and carries live in a fixed device array inside the
 * library (about 0.9 MB, held by every GPU that loads the library until
 * exit): at most 16384 tiles, i.e. n_rows + nnz <= 16384 * items_per_unit,
 * else FSB_ERR_LIMIT.  Calls whose kernels overlap on the GPU race on the
 * shared array.  The first call in a CUDA context (the device's primary
 * context, or a host framework's own context current on the calling thread)
 * resolves the array's address in that context and caches it per context;
 * that first call should come before any stream capture.                 */
int fsb_spmv_csr_noalloc(const fsb_csr* A, const void* x, void* y, int out_dtype,
                         int acc_mode, int32_t items_per_unit, void* stream);

/* y = A x.  out_dtype is value_dtype, or FSB_F32 for f16/bf16 values (the
 * precision form).  y must be zero-filled by the caller when row_map is set
 * (rows without a run are not written).
 * Replaces the launches of _spmv_csr_real_kernel / _spmv_csr_complex_kernel
 * (spmv_csr.py:677-705), the bucket kernels of
 * _triton_spmv_csr_impl_opt_prepared (spmv_csr.py:403-439) and the row-run
 * kernels _spmv_coo_seg_* (spmv_coo.py:436-478).                          */
int fsb_spmv_csr(const fsb_csr* A, const void* x, void* y, int out_dtype,
                 int acc_mode, const fsb_plan* plan, void* workspace,
                 int64_t workspace_bytes, void* stream);

/* C[:, :n_dense] = A B with B row-major (n_cols x n_dense, row stride ldb
 * elements) and C row-major (n_rows x n_dense, row stride ldc elements).
 * Replaces _spmm_csr_real/complex_kernel (spmm_csr.py:553-598), the opt
 * bucket and split kernels (spmm_csr.py:1252-1360), the alg2 kernels
 * (spmm_csr_opt_alg2.py:684-768) and the COO row-run kernels
 * (spmm_coo.py:415-460).                                                  */
int fsb_spmm_csr(const fsb_csr* A, const void* B, int64_t ldb, int64_t n_dense,
                 void* C, int64_t ldc, int out_dtype, int acc_mode,
                 const fsb_plan* plan, void* workspace, int64_t workspace_bytes,
                 void* stream);

/* Unsorted COO, one atomic add per product into a zero-filled y / C whose
 * element type acc_dtype is the value type or its wide type (f32 -> f64,
 * c64 -> c128); products are formed in acc_dtype.  Order not deterministic.
 * Replaces _spmv_coo_atomic_* (spmv_coo.py:229-294, launched at :451-491)
 * and _spmm_coo_atomic_* (spmm_coo.py:243-311, launched at :487-522).     */
int fsb_spmv_coo_atomic(const void* values, const void* row, const void* col,
                        int value_dtype, int index_dtype, int64_t nnz,
                        const void* x, void* y, int acc_dtype, void* stream);
int fsb_spmm_coo_atomic(const void* values, const void* row, const void* col,
                        int value_dtype, int index_dtype, int64_t nnz,
                        const void* B, int64_t ldb, int64_t n_dense, void* C,
                        int64_t ldc, int acc_dtype, void* stream);

/* offsets[b] = number of keys below b for b = 0 .. n_bins (n_bins + 1
 * entries) from nondecreasing keys in [0, n_bins): CSR row offsets of sorted
 * COO rows, column offsets of a transpose.  No host synchronisation (can be
 * captured in a CUDA graph); equals cumsum(bincount(keys)).  Replaces the
 * bincount + cumsum of coo_to_csr_for_spmv (spmv_csr.py:885-909) and
 * _transpose_csr_for_spmv (spmv_csr.py:456-494).                          */
int fsb_sorted_keys_to_offsets(const void* keys, int key_dtype, int64_t n,
                               int64_t n_bins, int64_t* offsets, void* stream);

/* ---- integer prepare steps ---------------------------------------------- *
 * Stable sort of n int32 / int64 keys (key_dtype FSB_I32 / FSB_I64):
 * keys_out (may be NULL) receives the keys in ascending order and
 * order_out[n] (int64) the permutation, ties in input order -- the same
 * result as torch.sort(keys, stable=True).  key_bits < the key width
 * promises keys in [0, 2^key_bits) (one 8-bit radix pass per started byte);
 * key_bits = the width sorts any values, signed.  n < 2^31.  Workspace:
 * fsb_sort_workspace_bytes(n, key_dtype, key_bits) bytes (-1 for bad
 * arguments).  Replaces the stable argsorts of _transpose_csr_for_spmv
 * (spmv_csr.py:456-494), coo_to_csr_for_spmv (spmv_csr.py:885-909) and
 * _sort_coo_lex_inplace (spmv_coo.py:297-309, spmm_coo.py:21-32).         */
int64_t fsb_sort_workspace_bytes(int64_t n, int key_dtype, int key_bits);
int fsb_stable_sort(const void* keys, int key_dtype, int64_t n, int key_bits,
                    void* keys_out, int64_t* order_out, void* workspace,
                    int64_t workspace_bytes, void* stream);

/* Starts of the runs of equal keys in n sorted int32 / int64 keys: starts
 * (capacity n + 1, int32 or int64 by starts_dtype) receives 0, the index of
 * every key that differs from its predecessor, and n; *count (device
 * int64) the number of entries written.  Replaces the nonzero-based
 * _seg_starts_from_sorted_rows (spmv_coo.py:312-327, spmm_coo.py:121-132).
 * Workspace: fsb_run_starts_workspace_bytes(n).                            */
int64_t fsb_run_starts_workspace_bytes(int64_t n);
int fsb_run_starts(const void* sorted_keys, int key_dtype, int64_t n,
                   void* starts, int starts_dtype, int64_t* count,
                   void* workspace, int64_t workspace_bytes, void* stream);

/* Duplicate merge of sorted COO entries (torch's coalesce, called by
 * FlagSparse's _coalesce_coo_entries, spmm_coo.py:35-51): with keys sorted
 * stably (fsb_stable_sort: sorted_keys, order) and their runs (fsb_run_starts:
 * starts, count), out_keys[j] = the j-th distinct key and out_values[j] =
 * the sum of its values in sorted order, from zero in float (half types,
 * float32), double (float64) or their pairs (complex), rounded once to the
 * value type; with n < 2 the value is copied unchanged.  out_keys /
 * out_values need room for n entries; *count - 1 of them are written (the
 * count stays on the device).                                             */
int fsb_coo_coalesce(const void* sorted_keys, int key_dtype,
                     const int64_t* order, const void* values,
                     int value_dtype, int64_t n, const void* starts,
                     int starts_dtype, const int64_t* count, void* out_keys,
                     void* out_values, void* stream);

/* ---- structured form: runs of consecutive columns and long rows -------- *
 * Descriptors added to a CSR matrix (which stays as it is) for the precision
 * form's SpMV / SpMM on matrices whose nonzeros sit mostly in runs of
 * consecutive columns (a band) or in a few long rows.  All device arrays.   */
typedef struct fsb_struct {
    const int32_t* run_col;   /* [n_rows] first column of the row's run       */
    const int32_t* run_off;   /* [n_rows] offset of the run inside the row    */
    const int32_t* run_len;   /* [n_rows] run length, 0: none, -1: long row   */
    const int64_t* tile_base; /* [ceil(n_rows / 128)] first column of the
                                 tile's run span                               */
    const int32_t* tile_span; /* [ceil(n_rows / 128)] span width, a multiple
                                 of 16, at most 256 (0: no runs)              */
    int32_t max_span;         /* largest tile_span                            */
    int32_t chunk_nnz;        /* SpMM: nonzeros per chunk of a long row       */
    int64_t n_long;           /* long rows                                    */
    const int32_t* long_rows; /* [n_long] their indices                       */
    int64_t n_chunks;         /* SpMM: chunks of the long rows                */
    const int32_t* chunk_row; /* [n_chunks] long-row position of each chunk   */
    const int64_t* chunk_ptr; /* [n_long + 1] first chunk of each long row    */
    int32_t xblock;           /* SpMV: columns of x per block (<= 65536)      */
    int32_t reserved;
    int64_t n_xblocks;        /* SpMV: ceil(n_cols / xblock)                  */
    const int64_t* seg_ptr;   /* [n_xblocks * n_long + 1] start of the (block,
                                 long row) segments of the regrouped nonzeros */
    const void* seg_val;      /* values of the long rows, by (block, row)     */
    const uint16_t* seg_off;  /* their columns minus the block's first column */
    /* SpMM, optional (lt_rec null: chunks): the long rows in tiles of
     * lt_rows rows x lt_cols columns (compiled: 512 x 1024).
     * Per (row group, column block) segment: records (value bits | column
     * inside the block << 16), ordered by row, padded to a multiple of 4,
     * starting at lt_seg_start (a multiple of 4), with lt_rows + 8 16-bit
     * per-row record starts (lt_rows + 1 used).                             */
    int64_t lt_groups;          /* ceil(n_long / lt_rows)                    */
    int64_t lt_col_blocks;      /* ceil(n_cols / lt_cols)                    */
    int32_t lt_rec_cap;         /* longest padded segment, in records        */
    int32_t lt_rows;
    int32_t lt_cols;
    int32_t reserved3;
    const uint32_t* lt_rec;
    const int64_t* lt_seg_start; /* [lt_groups * lt_col_blocks]              */
    const int32_t* lt_seg_len;   /* [lt_groups * lt_col_blocks] padded        */
    const uint16_t* lt_row_start;/* [lt_groups * lt_col_blocks * (lt_rows + 8)] */
} fsb_struct;

/* Per-row descriptors: the longest run of consecutive columns of each row of
 * at most long_min nonzeros (run_len < min_run: no run); longer rows get
 * run_len = -1.  No FlagSparse counterpart (FlagSparse buckets rows by length
 * only, spmv_csr.py:345-391, spmm_csr.py:444-477).                          */
int fsb_struct_rows(const fsb_csr* A, int64_t long_min, int32_t min_run,
                    int32_t* run_col, int32_t* run_off, int32_t* run_len,
                    void* stream);
/* Per-tile spans (tiles of 128 rows); runs that do not fit a 256-column span
 * starting at the tile's first run column are dropped (run_len, run_off set
 * to 0).                                                                    */
int fsb_struct_tiles(int64_t n_rows, const int32_t* run_col, int32_t* run_off,
                     int32_t* run_len, int64_t* tile_base, int32_t* tile_span,
                     void* stream);
/* Workspace bytes of fsb_struct_spmv (is_spmm 0) / fsb_struct_spmm.         */
int64_t fsb_struct_workspace_bytes(int is_spmm, const fsb_struct* S,
                                   int64_t n_dense);
/* y (float32) = A x, A and x float16 / bfloat16, float32 accumulation (long
 * rows compensated).  Replaces, for the precision form, the bucket kernels
 * of FlagSparse's opt SpMV (spmv_csr.py:393-440).                           */
int fsb_struct_spmv(const fsb_csr* A, const fsb_struct* S, const void* x,
                    float* y, void* workspace, int64_t workspace_bytes,
                    void* stream);
/* C (float32) = A B, B row-major float16 / bfloat16 with n_dense of 16, 32
 * or 64; runs on the tensor cores (tcgen05, float32 accumulators in tensor
 * memory), long rows in chunks (compensated).  B and C 16-byte aligned, ldb
 * a multiple of 8, ldc of 4.  Replaces, for the precision form, the bucket
 * and split kernels of FlagSparse's opt SpMM (spmm_csr.py:1252-1360).       */
int fsb_struct_spmm(const fsb_csr* A, const fsb_struct* S, const void* B,
                    int64_t ldb, int64_t n_dense, float* C, int64_t ldc,
                    void* workspace, int64_t workspace_bytes, void* stream);

/* ---- block-sparse SpMM on the tensor cores ----------------------------- *
 * C (float32, n_rows x n_dense, row stride ldc) = A B for A in BSR form with
 * dense 16 x 16 blocks: block_values[n_blocks][16][16] (row-major blocks,
 * bf16 or f16: value_dtype = FSB_BF16 / FSB_F16), block_col[n_blocks] (block
 * columns), block_row_ptr[ceil(n_rows / 16) + 1]; B (n_cols x n_dense, row
 * stride ldb) has the same 16-bit type, is 16-byte aligned, with ldb and
 * n_dense multiples of 8.  tcgen05.mma (kind::f16, fp32 accumulation in
 * tensor memory), one MMA of 128 x 16 x 16 per stored block and 128-column
 * tile; n_blocks = block_row_ptr's last entry.  staging:
 * FSB_BSR_STAGE_TMA stages B slices and blocks with the Tensor Memory
 * Accelerator (tensor maps, 4-stage ring run by one thread;
 * FSB_ERR_UNSUPPORTED when no tensor map can be encoded),
 * FSB_BSR_STAGE_THREADS with the CTA's threads.  No FlagSparse counterpart: FlagSparse runs
 * block-structured matrices through its CSR SpMM (spmm_csr.py:2088-2157).  */
#define FSB_BSR_STAGE_TMA     0
#define FSB_BSR_STAGE_THREADS 1
int fsb_bsr_spmm_tc(const void* block_values, int value_dtype,
                    const void* block_col, int index_dtype,
                    const void* block_row_ptr, int ptr_dtype, int64_t n_rows,
                    int64_t n_cols, int64_t n_blocks, const void* B,
                    int64_t ldb, int64_t n_dense, float* C, int64_t ldc,
                    int staging, void* stream);

/* ---- SDDMM ------------------------------------------------------------- *
 * out[p] = alpha * dot(x[row_ids[p]], y[col_idx[p]]) + beta * data[p] for
 * the nnz stored positions of a CSR pattern (data may be null: beta term
 * dropped); x (n_rows x k, row stride ldx) and y (n_cols x k, row stride
 * ldy) row-major, float32 (float32 accumulation) or float64.  Replaces the
 * launch of _sddmm_csr_real_kernel in _run_sddmm_prepared
 * (sddmm_csr.py:271-348).                                                  */
int fsb_sddmm_csr(const void* col_idx, int index_dtype, const int32_t* row_ids,
                  int64_t nnz, int64_t n_rows, int64_t n_cols, const void* x,
                  int64_t ldx, const void* y, int64_t ldy, int64_t k,
                  const void* data, void* out, int value_dtype, double alpha,
                  double beta, void* stream);

/* ---- diagnostic SpMM forms ------------------------------------------ *
 * C = A B with a fixed-order, explicitly rounded accumulation per element,
 * the arithmetic of FlagSparse's diagnose-only SpMM paths (stable kernels
 * spmm_csr.py:922-1249, candidate short-row kernels :1501-1634, entry
 * points :1998-2086).  Each output element walks its row's nonzeros in
 * order:
 *   FSB_DIAG_NATIVE      acc = fma(a, b, acc), value precision
 *   FSB_DIAG_WIDE        acc = fma(a, b, acc) in float64, stored in the
 *                        value type (float64 accumulate, float32 store)
 *   FSB_DIAG_KAHAN       y = fma(a, b, -comp); t = acc + y;
 *                        comp = (t - acc) - y; acc = t, value precision
 *   FSB_DIAG_KAHAN_WIDE  the same in float64, stored in the value type
 * Rows of at most short_max nonzeros use mode_short, the others mode_long.
 * float32 / float64 values; B (ldb) and C (ldc) row-major, C in the value
 * type.  For diagnosis, not speed: one warp per row.                      */
#define FSB_DIAG_NATIVE     0
#define FSB_DIAG_WIDE       1
#define FSB_DIAG_KAHAN      2
#define FSB_DIAG_KAHAN_WIDE 3
int fsb_spmm_csr_diag(const fsb_csr* A, const void* B, int64_t ldb,
                      int64_t n_dense, void* C, int64_t ldc, int mode_short,
                      int mode_long, int64_t short_max, void* stream);

/* ---- Matrix Market ingest (host) ------------------------------------- *
 * Parses a .mtx coordinate file into CSR (float64 values, int64 indices and
 * row offsets, columns sorted in each row) with the semantics of FlagSparse's
 * loader load_mtx_to_csr_torch (tests/test_spmv.py:103-178): pattern
 * entries 1.0, duplicates summed in file order, symmetric / hermitian
 * entries mirrored, skew-symmetric ones mirrored negated, out-of-range
 * entries dropped.  fsb_mtx_open parses (threads <= 0: all host threads) and
 * returns a handle (null on error, message in fsb_last_error) with the sizes;
 * fsb_mtx_read copies into caller arrays of n_rows + 1 / nnz / nnz entries;
 * fsb_mtx_close frees the handle.  No GPU involved.                       */
void* fsb_mtx_open(const char* path, int64_t* n_rows, int64_t* n_cols,
                   int64_t* nnz, int threads);
int   fsb_mtx_read(void* handle, int64_t* indptr, int64_t* indices,
                   double* values);
void  fsb_mtx_close(void* handle);

/* ---- learned plan selector -------------------------------------------- *
 * No FlagSparse counterpart: FlagSparse picks its launch parameters by
 * fixed row-length buckets and device-property heuristics
 * (spmm_csr.py:395-414, spmm_csr_opt_alg2.py:175-304).  These entry points
 * are the device side of the learned selector that replaces them.         */

/* Structure features of a CSR matrix (six doubles, zeroed by the caller,
 * accumulated on stream): out[0] = sum of row lengths, out[1] = sum of
 * squared row lengths, out[2] = longest row (an unsigned 64-bit integer
 * held in the slot's bits), out[3] = empty rows, out[4] = sum over nonzeros
 * of |col - r * n_cols / n_rows| / n_cols, out[5] = nonzeros whose column
 * and position in the row agree modulo 16 (all of them when the rows are
 * aligned dense 16-column blocks).  Sums of doubles are accumulated with
 * atomics (last-bit order dependence).                                    */
int fsb_csr_features(const void* row_ptr, int ptr_dtype, const void* col_idx,
                     int index_dtype, int64_t n_rows, int64_t n_cols,
                     double* out, void* stream);

/* The selector network: d_in -> h1 (ReLU) -> h2 (ReLU) -> d_out, float32,
 * parameters packed W1[d_in][h1], b1, W2[h1][h2], b2, W3[h2][d_out], b3
 * (d_in <= 16, h1, h2 <= 64, d_out <= 32).  Returns the parameter count.  */
int fsb_mlp_param_count(int d_in, int h1, int h2, int d_out);

/* Y[n][d_out] = network(X[n][d_in]).  cache (may be null) receives per
 * sample the pre-activations Z1[h1], Z2[h2] and Y[d_out].                 */
int fsb_mlp_forward(const float* X, int n, int d_in, int h1, int h2,
                    int d_out, const float* params, float* Y, float* cache,
                    void* stream);

/* Gradient of L = inv_terms * sum mask (Y - T)^2 with respect to the
 * parameters, from a forward cache: grad (packed like params) is written
 * with fixed-order sums over the samples; loss_terms[n] receives each
 * sample's sum of masked squared errors; deltas is n x (h1 + h2 + d_out)
 * scratch.                                                                 */
int fsb_mlp_backward(const float* X, int n, int d_in, int h1, int h2,
                     int d_out, const float* params, const float* cache,
                     const float* targets, const float* mask, float inv_terms,
                     float* deltas, float* loss_terms, float* grad,
                     void* stream);

/* One Adam step (Kingma & Ba, bias-corrected, step >= 1); weight_decay
 * adds weight_decay * p to the gradient (L2 regularisation).              */
int fsb_adam_step(float* params, const float* grad, float* m1, float* m2,
                  int n_params, float lr, float beta1, float beta2, float eps,
                  int step, float weight_decay, void* stream);

/* ---- measurement: the gather floor of an SpMM ---------------------------
 * No counterpart in FlagSparse: a roofline probe for the SpMM kernels.
 * Gathers, for each of the nnz column indices col_idx[k] (int32, each in
 * [0, rows of B)), the float32 row B[col_idx[k]][0 .. n_dense) (n_dense 32,
 * 64 or 128, 16-byte aligned rows of stride ldb) exactly as the product
 * kernels do, and adds them into per-thread sums written to out (at least
 * SMs x 16 x 128 floats).  Nothing else is computed, so its time on a
 * matrix is the speed limit of any product that reads one B row per
 * nonzero.  variant in [0, FSB_GATHER_FLOOR_VARIANTS): gathers in flight per
 * lane x resident warps (4 x 64, 8 x 32, 16 x 16, 6 x 48 per SM).          */
#define FSB_GATHER_FLOOR_VARIANTS 4
int fsb_gather_floor(const int32_t* col_idx, int64_t nnz, const float* B,
                     int64_t ldb, int64_t n_dense, float* out,
                     int64_t out_len, int variant, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* FLAGSPARSE_B200_H */
