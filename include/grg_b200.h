/*
 * grg_b200.h - C ABI of the B200 GRG matmul backend (libgrg_b200.so).
 *
 * The library computes the GRG "up" (X*G, samples -> mutations) and "down" (X*G^T,
 * mutations -> samples) traversals on one NVIDIA B200 (sm_100a).  All entry points take
 * plain device/host pointers, sizes and a cudaStream_t; none allocates device memory: the
 * caller (the Python runtime, via PyTorch) owns every buffer.  Every function returns a
 * grg_b200_status; grg_b200_last_error() gives the message of the last failure on the
 * calling thread.  Launches are asynchronous on the given stream and may be captured in a
 * CUDA graph.
 *
 * Replaced reference interfaces (paths inside CornellHPC/grg-spmv):
 *   grg_b200_traverse      - the whole prepared call: TritonRuntime._execute_prepared
 *                            (pygrgl_spmv/backends/triton/backend.py:1221-1225), i.e.
 *                            _seed_state (:1116-1150), _enqueue_wavefront (:970-1049) with
 *                            launch_block / csr_spmm_add_kernel / csc_spmm_add_kernel
 *                            (pygrgl_spmv/backends/triton/kernel.py:57-206), and
 *                            _write_output (:1178-1219) with _apply_endpoint_bias (:1152-1176);
 *                            the cuSPARSE equivalent is CusparseRuntime._seed_prepared,
 *                            _enqueue_wavefront, _write_prepared_output
 *                            (pygrgl_spmv/backends/cusparse/backend.py:1633-1828).
 *   grg_b200_seed_up       - the up branch of _seed_state (triton/backend.py:1120-1141).
 *   grg_b200_run_level     - one destination level of _enqueue_wavefront: every
 *                            launch_block call of that level fused into one gather pass
 *                            (triton/backend.py:1030-1046); for down it also performs the
 *                            selector scatter of _seed_state (:1143-1150) as a gather.
 *   grg_b200_output_up     - the up branch of _write_output (triton/backend.py:1189-1210).
 *   grg_b200_output_down   - the down branch of _write_output (triton/backend.py:1212-1219).
 *   grg_b200_emit_all      - the emit_all_nodes branch of _write_output (:1185-1187).
 *   grg_b200_ring_create / grg_b200_ring_destroy
 *                          - the per-slot copy streams and events of the streamed ring
 *                            (triton/backend.py:710, :738-746, :958-968).
 *   grg_b200_last_error    - error reporting (the Python side raises RuntimeError with it).
 *
 * Data layout (all ids are positions in the artifact's stable height order):
 *   state   [num_nodes, ld_state]     node values, row-major
 *   input   [rows, ld_input]          up: samples (or individuals), down: mutations
 *   output  [rows, ld_output]         up: mutations, down: samples (or individuals),
 *                                     emit_all_nodes: all nodes in ORIGINAL node order
 *   level   a gather list per destination row: the row's value is
 *             init(row) + seg_1 + seg_2 + ...   (left to right)
 *           where each segment is a sum, from zero and in list order, of the entries that
 *           follow a GRG_B200_SEG_START-flagged entry.  An entry names a state row, an
 *           input row or a miss row (GRG_B200_SRC_*).  This reproduces the accumulation
 *           order of the reference's ReferenceRuntime (per source level, one sparse product
 *           added to the destination; pygrgl_spmv/backends/reference.py:396-429).
 */
#ifndef GRG_B200_H
#define GRG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GRG_B200_ABI_VERSION 14

typedef enum grg_b200_status {
    GRG_B200_OK = 0,
    GRG_B200_ERR_INVALID = 1,     /* bad argument; nothing was launched */
    GRG_B200_ERR_CUDA = 2,        /* a CUDA runtime call failed */
    GRG_B200_ERR_UNSUPPORTED = 3  /* valid request outside the library's limits */
} grg_b200_status;

/*
 * GRG_B200_MIXED: input, output, miss and init buffers are FP64; the node state (and, for
 * down, encoded copies of input and miss in mix_scratch) is stored in 6 bytes per value:
 * hi = the value rounded to FP32 and lo = a 16-bit correction in units of 2^(e(hi) - 38), so
 * a stored value is within 2^-39 of the exact one relative to |hi| (integers below 2^39 are
 * exact).  Sums are accumulated in FP64 and rounded back once per node.  A mixed buffer of
 * R rows and ld columns (ld a multiple of 4) is float hi[R * ld] followed by int16
 * lo[R * ld]; see GRG_B200_MIX_BYTES.  Mixed traversals never use exact order.
 */
typedef enum grg_b200_dtype { GRG_B200_F64 = 0, GRG_B200_F32 = 1, GRG_B200_MIXED = 2 } grg_b200_dtype;

/* Bytes of one mixed buffer of `rows` rows and `ld` columns (each plane rounded up to 16). */
#define GRG_B200_MIX_PLANE(bytes) ((((bytes) + 15) / 16) * 16)
#define GRG_B200_MIX_BYTES(rows, ld) \
    (GRG_B200_MIX_PLANE((int64_t)(rows) * (ld) * 4) + GRG_B200_MIX_PLANE((int64_t)(rows) * (ld) * 2))
typedef enum grg_b200_direction { GRG_B200_UP = 0, GRG_B200_DOWN = 1 } grg_b200_direction;
typedef enum grg_b200_init {
    GRG_B200_INIT_NONE = 0,
    GRG_B200_INIT_VECTOR = 1,  /* every node starts at init_vector[col] */
    GRG_B200_INIT_XTX = 2,     /* every node starts at xtx_node[row] (2 * coalescence count) */
    GRG_B200_INIT_MATRIX = 3   /* node row starts at init_matrix[node_perm[row], col] */
} grg_b200_init;
typedef enum grg_b200_bias {
    GRG_B200_BIAS_NONE = 0,
    GRG_B200_BIAS_VECTOR = 1,  /* out[r, c] += bias[r] * init_vector[c] (product rounded first) */
    GRG_B200_BIAS_XTX = 2      /* out[r, c] += bias[r] */
} grg_b200_bias;

/* Gather-list entry coding (uint32). */
#define GRG_B200_SEG_START 0x80000000u
#define GRG_B200_SRC_SHIFT 29
#define GRG_B200_SRC_MASK 0x3u
#define GRG_B200_SRC_STATE 0u /* id = state row */
#define GRG_B200_SRC_INPUT 1u /* id = input row (down: mutation) */
#define GRG_B200_SRC_MISS 2u  /* id = miss row (down: mutation), skipped unless use_miss */
#define GRG_B200_SRC_NULL 3u  /* padding entry: skipped, never flagged as a segment start */
#define GRG_B200_ID_MASK 0x1FFFFFFFu
#define GRG_B200_MAX_ID 0x1FFFFFFFu

/*
 * One destination level.  Its gather structure is one byte blob with these arrays at
 * 16-byte aligned offsets.  Rows are stored in *processing order* (chosen on the host for
 * cache locality); processing position p computes level-local row row_ids[p] (or p itself
 * when off_row_ids < 0).  Rows with more than heavy_threshold entries are the last num_heavy
 * positions (split across a warp or a CTA per row, heavy_variant); narrow kernels cover the
 * first num_rows - num_heavy:
 *   int32  row_ptr[num_rows + 1]     entry offsets of each processing position
 *   int32  heavy_rows[num_heavy]     the heavy positions (num_rows - num_heavy, ...)
 *   int32  row_ids[num_rows]         optional processing position -> level-local row
 *   uint32 entries[num_entries]
 * list_align = 4: every position's list starts at a multiple of 4 entries and holds a
 * multiple of 4 entries (null-padded), so kernels may read 4 codes with one 16-byte load
 * (narrow variant 6 requires it); list_align = 1: no padding.
 * ring_slot < 0: blob is device memory.  ring_slot >= 0: blob is pinned host memory that
 * grg_b200_traverse copies into ring slot `ring_slot` before the level runs.
 */
/* Slot layout: the narrow rows form buckets of consecutive positions whose lists all hold the
 * same number of 4-entry quads, so a kernel computes a row's list from its position
 * (slot_entry[b] + (p - slot_pos[b]) * 4 * slot_width[b]) instead of loading row_ptr. */
#define GRG_B200_MAX_SLOT_BUCKETS 8

typedef struct grg_b200_level {
    int64_t row_begin;
    int64_t num_rows;
    int64_t num_entries;
    int64_t num_heavy;
    int32_t heavy_threshold;
    int32_t ring_slot;
    const void* blob;
    int64_t blob_bytes;
    int64_t off_row_ptr;
    int64_t off_heavy;
    int64_t off_row_ids; /* -1: identity order */
    int64_t off_entries;
    int32_t list_align;  /* 1 or 4 */
    int32_t num_slot_buckets; /* 0, or the slot layout of the narrow rows (list_align 4): */
    int64_t slot_pos[GRG_B200_MAX_SLOT_BUCKETS];   /* first processing position of bucket b */
    int64_t slot_entry[GRG_B200_MAX_SLOT_BUCKETS]; /* first entry of bucket b */
    int32_t slot_width[GRG_B200_MAX_SLOT_BUCKETS]; /* entries per row of bucket b, in quads of 4 */
    int64_t short_rows; /* the last short_rows narrow positions (those ending at num_rows -
                           num_heavy) hold at most 4 entries each: narrow variants 13 and 14 walk
                           them with one entry slot, twice the rows per CTA.  A speed hint:
                           longer lists there still sum correctly.  0 <= short_rows <=
                           num_rows - num_heavy; 0 for none. */
} grg_b200_level;

typedef struct grg_b200_ring grg_b200_ring; /* opaque: copy stream + per-slot events */

typedef struct grg_b200_traverse_args {
    int32_t dtype;        /* grg_b200_dtype */
    int32_t direction;    /* grg_b200_direction */
    int32_t init_mode;    /* grg_b200_init (applied inside the traversal) */
    int32_t bias_mode;    /* grg_b200_bias (applied to the output) */
    int32_t emit_all_nodes;
    int32_t by_individual;
    int32_t use_miss;     /* down: read miss rows; up: write miss output */
    int32_t exact_order;  /* 1: heavy rows also sum in list order (bit-exact with the reference) */
    int64_t k;
    int64_t num_nodes;
    int64_t num_samples;
    int64_t num_mutations;
    int64_t num_individuals;
    void* state;
    int64_t ld_state;
    const void* input;
    int64_t ld_input;
    void* output;
    int64_t ld_output;
    void* miss; /* down: miss input [M, ld_miss]; up: miss output [M, ld_miss] */
    int64_t ld_miss;
    const void* init_vector;            /* [k] */
    const void* init_matrix;            /* [num_nodes, ld_init], original node order */
    int64_t ld_init;
    const int32_t* node_perm;           /* [num_nodes] stable position -> original id */
    const int32_t* inv_node_perm;       /* [num_nodes] original id -> stable position */
    const void* xtx_node;               /* [num_nodes] 2 * coalescence count, stable order */
    const void* endpoint_bias;          /* up: [num_mutations], down: [num_samples] */
    const int32_t* sample_to_individual;/* up by_individual: [num_samples] */
    const int32_t* ind_ptr;             /* down by_individual: [num_individuals + 1] */
    const int32_t* ind_samples;         /* down by_individual: samples of each individual, ascending */
    const int32_t* sel_mut_ptr;         /* up: [num_mutations + 1] */
    const int32_t* sel_mut_idx;         /* up: node of each selector entry, stored order */
    const int32_t* sel_miss_ptr;
    const int32_t* sel_miss_idx;
    int64_t level0_rows;                /* up: number of level-0 rows to seed */
    int32_t num_levels;                 /* levels in execution order */
    const grg_b200_level* levels;
    grg_b200_ring* ring;                /* required when any level is streamed */
    void* const* slot_buffers;          /* device ring slots */
    const int64_t* slot_bytes;
    int32_t num_slots;
    int32_t* error_word;                /* optional device int32: first failed bounds check */
    int32_t narrow_variant;             /* narrow-row kernel shape, 0..GRG_B200_NARROW_VARIANTS-1:
                                           0: 4 rows per round; 1: 8 rows per round; 2: 4 rows per
                                           round from a shared-memory staged list; 3: 16 rows per
                                           round, staged; 4: cp.async gathers into shared memory,
                                           then in-order sums; 5: as 0 with at most 32 registers
                                           per thread (8 CTAs per SM); 6: padded lists (list_align
                                           4) read 4 codes per 16-byte load, next 4 prefetched
                                           while the current 4 rows load; 7: as 6 with 48
                                           registers per thread (5 CTAs per SM) instead of 40;
                                           8: as 6 with 8 codes (two 16-byte loads) and 8 row
                                           fetches in flight per round (3 CTAs per SM); 9: as 7,
                                           persistent: the narrow CTAs are capped at the resident
                                           count and each warp walks row groups, loading the next
                                           group's row pointers and first codes while the current
                                           rows load; 10: as 9 with 64 registers (4 CTAs per SM);
                                           11: as 7 with a lean walk for launches without an
                                           error word (no bounds checks, 32 x 32-bit row
                                           addressing, state-only decode on up levels, heavy rows
                                           likewise), bit-identical to 7; 12: as 11 but a row's
                                           entries are summed left to right into one partial sum
                                           (no per-segment restarts; default mode only);
                                           13: as 12 with entry-parallel narrow rows: a row's
                                           lanes form two entry slots, each lane adding one
                                           32-byte chunk of every other entry (k = 2^n x the
                                           vector width, no init, 32-byte aligned buffers;
                                           otherwise as 12); 14: as 13 with the codes of a row's
                                           first 4 quads loaded before the previous level ends.
                                           At k = V (k below a 32-byte chunk: k = 1, 2 in FP64)
                                           13 and 14 walk one V-column chunk lane per row;
                                           15 and 16: as 14 in 4-warp and 2-warp CTAs.
                                           13 and 14 walk a level's short_rows with one entry
                                           slot (each lane adds its chunk of all 4 entries).
                                           11 to 14 fall back to 7 with an
                                           error word, split rows or exact order.  Up level
                                           lists name state rows and null padding only. */
    int32_t heavy_variant;              /* heavy-row kernel outside exact order: 0 one CTA per row
                                           (list staged in shared memory, tree reduction); 1 one
                                           warp per row (lane groups split the list, shuffle
                                           reduction); 2 as 1 but in the same launch as the narrow
                                           rows (narrow_variant 6 to 10 only; otherwise as 1); 3 as 1
                                           with 32 heavy rows (1024 threads) per CTA.  Exact
                                           order always uses one CTA per row. */
    void* mix_scratch;                  /* GRG_B200_MIXED down: room for the encoded input, then
                                           (use_miss) the encoded miss rows, each a mixed buffer of
                                           num_mutations rows and ld_state columns */
    int64_t mix_scratch_bytes;
    int32_t narrow_split;               /* narrow_variant 6 to 10, default mode, FP64/FP32: split each narrow
                                           row over 2^narrow_split lane groups (0..3), or -1 to choose
                                           per level (long rows in levels too small to fill the GPU) */
    int32_t schedule;                   /* grg_b200_schedule */
    void* dataflow_sync;                /* GRG_B200_SCHEDULE_DATAFLOW and fused level runs: device int32[4], 16-byte aligned;
                                           [2] holds GRG_B200_DEVICE_WAIT_TIMEOUT after a failed wait */
    int32_t launch_flags;               /* GRG_B200_LAUNCH_* bits */
    int32_t persist_ctas;               /* narrow_variant 9/10: CTAs of a level launch's persistent
                                           narrow part (each loops over row groups); 0 = what the
                                           GPU holds at once (SMs x CTAs per SM) */
    int64_t fuse_entries;               /* > 0 (default mode, FP64/FP32, narrow_variant 6/7/9/10,
                                           heavy_variant 2, dataflow_sync set): runs of 2 to 48
                                           consecutive resident levels of at most this many entries
                                           each run as one cooperative launch with a bounded grid
                                           barrier between levels (results bit-identical; a barrier
                                           that gives up leaves GRG_B200_DEVICE_WAIT_TIMEOUT in
                                           dataflow_sync[2]); 0 = one launch per level */
} grg_b200_traverse_args;

/* Level, seed and output launches of the default kernels use programmatic dependent launch:
 * each may start while the previous kernel of the stream finishes, reads only the static
 * level lists until the hardware reports that kernel complete, and so overlaps the launch
 * gap.  Ignored when any level is streamed. */
#define GRG_B200_LAUNCH_PDL 1

/*
 * GRG_B200_SCHEDULE_LEVELS: one launch per level (each level waits for the previous one).
 * GRG_B200_SCHEDULE_DATAFLOW: one persistent launch for all levels of a traversal; a row
 * waits only for its own source rows.  Used when the call is in the default (not exact)
 * mode, FP64/FP32, every level resident with padded lists and at most 128 levels; other
 * calls run level by level.  The rows it writes are first filled with a NaN sentinel (a
 * quiet NaN with payload 0x80DEADBEEF001 for FP64, 0x40DEAD for FP32): inputs holding that
 * exact NaN make the wait time out (status GRG_B200_DEVICE_WAIT_TIMEOUT, result undefined).
 */
typedef enum grg_b200_schedule { GRG_B200_SCHEDULE_LEVELS = 0, GRG_B200_SCHEDULE_DATAFLOW = 1 } grg_b200_schedule;
#define GRG_B200_DEVICE_WAIT_TIMEOUT 6

#define GRG_B200_NARROW_VARIANTS 17

/* Library ABI version (GRG_B200_ABI_VERSION of the build). */
int grg_b200_abi_version(void);

/* Copies the last error message of the calling thread into buf (always NUL-terminated). */
size_t grg_b200_last_error(char* buf, size_t buf_size);

/* Ring of streamed-structure slots: one non-blocking copy stream on `device` and two events
 * per slot.  Replaces the Triton runtime's slot copy streams and copy/compute events. */
int grg_b200_ring_create(int device, int num_slots, grg_b200_ring** out);
int grg_b200_ring_destroy(grg_b200_ring* ring);

/* Seeds level 0 of an up traversal: state[r] = init(r) (+ input[r or sample_to_individual[r]]
 * for r < num_samples).  Uses dtype, init_mode, by_individual, k, the state/input/init fields
 * and level0_rows of args. */
int grg_b200_seed_up(const grg_b200_traverse_args* args, void* stream);

/* Runs one destination level (narrow rows, then heavy rows).  The level's blob must already
 * be device-resident (slot < 0) or copied (blob then names the device copy). */
int grg_b200_run_level(const grg_b200_traverse_args* args, const grg_b200_level* level, void* stream);

/* Up outputs: output[m] = sum of state rows of sel_mut row m (stored order) + endpoint bias;
 * with use_miss also miss[m] from sel_miss (no bias). */
int grg_b200_output_up(const grg_b200_traverse_args* args, void* stream);

/* Down output: output[s] = state[s] + bias[s], or with by_individual
 * output[i] = sum over the individual's samples (ascending) of (state[s] + bias[s]). */
int grg_b200_output_down(const grg_b200_traverse_args* args, void* stream);

/* All-node output in original order: output[j] = state[inv_node_perm[j]]. */
int grg_b200_emit_all(const grg_b200_traverse_args* args, void* stream);

/* The full prepared call: seed, every level (copying streamed levels through the ring), and
 * the output stage, all on `stream`. */
int grg_b200_traverse(const grg_b200_traverse_args* args, void* stream);

/*
 * Row-wise step of the standardised genotype Gram operators (Z^T Z and Z Z^T with Z centred by
 * the allele mean and scaled by 1/sigma per mutation): the FP64 work between and after the two
 * traversals, fused into one pass over a [rows, k] buffer (row stride ld for every buffer).
 * Replaces the CuPy/cuBLAS steps of the reference's PreparedXTX._body
 * (scripts/pca_bench/__main__.py:326-347) and its row_weighted_sum kernel (:32-61), and the
 * kinship product of scripts/bolt_lmm_inf/core.py:1241-1301.  Per row r and column j:
 *     t = src[r, j]
 *     if miss_in:    t = t + miss_in[r, j] * miss_scale[r]
 *     if pre_scale:  t = t * pre_scale[r]
 *     if col_sub:    t = t - col_sub[j] * (sub_scale ? sub_scale[r] : 1)
 *     if post_scale: t = t * post_scale[r]
 *     dst[r, j] = t;  if miss_out: miss_out[r, j] = t * miss_out_scale[r]
 *     if col_sums:   sums[j] = sum over r of t * (sum_weight ? sum_weight[r] : 1)
 * Every product and sum is rounded separately (no fused multiply-add).  The column sums are
 * deterministic: fixed row blocks, a fixed in-block order, then the blocks' partials in block
 * order (partials needs GRG_B200_ROWOP_BLOCKS(rows) * k doubles, each row block a contiguous
 * range of ceil(rows / blocks) rows).  src may equal dst and
 * miss_in may equal miss_out (each element is read before it is written, by one thread).
 */
typedef struct grg_b200_rowop_args {
    int64_t rows;
    int64_t k;
    int64_t ld;
    const double* src;
    double* dst;
    const double* miss_in;
    const double* miss_scale;
    const double* pre_scale;
    const double* col_sub;
    const double* sub_scale;
    const double* post_scale;
    double* miss_out;
    const double* miss_out_scale;
    int32_t col_sums;
    const double* sum_weight;
    double* partials;
    double* sums;
} grg_b200_rowop_args;

/* Row blocks of a rowop call: one per 256 rows, at most 1184 (the partial sums hold one row of
 * k doubles per block). */
#define GRG_B200_ROWOP_MAX_BLOCKS 1184
#define GRG_B200_ROWOP_BLOCKS(rows) \
    ((((rows) + 255) / 256) < GRG_B200_ROWOP_MAX_BLOCKS ? (((rows) + 255) / 256) : GRG_B200_ROWOP_MAX_BLOCKS)
int grg_b200_rowop(const grg_b200_rowop_args* args, void* stream);

/* No counterpart in the reference.  The same traversal as grg_b200_traverse for callers that
 * cannot allocate device memory (C/FFI hosts without a device allocator, plugins inside
 * another framework's memory manager, code that must not allocate during stream capture):
 * args->state and args->ld_state are ignored and the node state is kept in a fixed array of
 * GRG_B200_STATIC_STATE_BYTES inside this library, which every GPU that loads the library
 * holds until the process exits.  The caller still passes inputs, outputs and level blobs.
 *   - num_nodes * k * sizeof(element) must not exceed GRG_B200_STATIC_STATE_BYTES, and every
 *     level must be resident (ring_slot < 0); otherwise GRG_B200_ERR_UNSUPPORTED.
 *   - The first call on a device looks up the array's device address (cudaGetSymbolAddress,
 *     once per device, with that device current); make that first call before any stream
 *     capture that will contain the entry point.  The address is kept per device and driver
 *     context: after cudaDeviceReset, or from a context the caller created itself, the next
 *     call looks it up again (that call, too, belongs outside a capture).
 *   - All calls share the one array: calls whose work overlaps on the GPU (different streams,
 *     no ordering between them) race on it.  Calls ordered on one stream are safe; every
 *     traversal writes each node row before reading it, so nothing needs clearing. */
#define GRG_B200_STATIC_STATE_BYTES (16u << 20)
int grg_b200_traverse_static(const grg_b200_traverse_args* args, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GRG_B200_H */
