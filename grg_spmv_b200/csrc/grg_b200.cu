// libgrg_b200: GRG up/down traversal kernels for NVIDIA B200 (sm_100a) behind a C ABI.
//
// The operand of a GRG traversal is a 0/1 DAG, so each level is a gather-sum: every
// destination row adds up the rows it points at.  There is no dense contraction, so the
// tensor cores have nothing to do; the kernels are bound by HBM/L2 traffic (the gather list
// is streamed once, node rows are read once per edge and written once).  Design:
//
//  * One pass per destination level, atomic-free: up gathers each node's children, down
//    gathers each node's parents (the reference's Triton CSC kernel scatters with atomics
//    instead, pygrgl_spmv/backends/triton/kernel.py:101-138).  Results are deterministic.
//  * Narrow rows: a group of G lanes owns one row; each lane holds V consecutive columns
//    (double2 / float4 vector loads), so a warp covers 32/G rows and the k columns of a row
//    are read as one contiguous segment.  The lane sums the row's list left to right, one
//    segment at a time, exactly like ReferenceRuntime (one sparse product per source level
//    added to the destination, pygrgl_spmv/backends/reference.py:396-429).
//  * Heavy rows (more than heavy_threshold entries; down-direction samples can have
//    thousands of parents) get one 128-thread CTA each.  Default: entries are split over
//    the CTA and tree-reduced in a fixed order (deterministic, exact for integer-valued
//    inputs).  exact_order=1: the CTA loads chunks in parallel and one thread group adds them
//    in list order, which is bit-identical to the reference for any input.
//  * Down seeding (sel_mut^T x and sel_miss^T miss, the reference's atomic index_add_ at
//    triton/backend.py:1143-1150) is folded into the level lists as leading INPUT/MISS
//    segments, so it costs no extra pass; up seeding touches level 0 only.
//  * Streamed levels are copied from pinned host memory into device ring slots on a copy
//    stream, ordered with per-slot events, so copies overlap the previous levels' compute.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <type_traits>

#include "grg_b200.h"

namespace {

thread_local char g_last_error[1024] = "";

int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return code;
}

#define GRG_CUDA_TRY(expr)                                                                  \
    do {                                                                                    \
        cudaError_t err__ = (expr);                                                         \
        if (err__ != cudaSuccess)                                                           \
            return fail(GRG_B200_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(err__)); \
    } while (0)

#define GRG_LAUNCH_CHECK(name)                                                              \
    do {                                                                                    \
        cudaError_t err__ = cudaGetLastError();                                             \
        if (err__ != cudaSuccess)                                                           \
            return fail(GRG_B200_ERR_CUDA, "launch of %s failed: %s", name, cudaGetErrorString(err__)); \
    } while (0)

// Launch with programmatic dependent launch when `pdl` (the kernel must call pdl_wait()
// before touching data that earlier kernels of the stream produce).
template <typename... KArgs, typename... Args>
cudaError_t launch_k(bool pdl, cudaStream_t s, dim3 grid, int block, void (*kernel)(KArgs...), Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(static_cast<unsigned>(block));
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = pdl ? attr : nullptr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// ---------------------------------------------------------------------------------------
// Vector packs
// ---------------------------------------------------------------------------------------
template <typename T, int V>
struct alignas(sizeof(T) * V) Pack {
    T v[V];
};

template <typename T, int V>
__device__ __forceinline__ Pack<T, V> zero_pack() {
    Pack<T, V> r;
#pragma unroll
    for (int i = 0; i < V; ++i) r.v[i] = T(0);
    return r;
}

template <typename T, int V>
__device__ __forceinline__ Pack<T, V> splat(T x) {
    Pack<T, V> r;
#pragma unroll
    for (int i = 0; i < V; ++i) r.v[i] = x;
    return r;
}

template <typename T, int V>
__device__ __forceinline__ void add_into(Pack<T, V>& a, const Pack<T, V>& b) {
#pragma unroll
    for (int i = 0; i < V; ++i) a.v[i] = a.v[i] + b.v[i];
}

// Read-only (non-coherent) load: every row read by a kernel was written by an earlier launch.
template <typename T, int V>
__device__ __forceinline__ Pack<T, V> ld_ro(const T* p) {
    Pack<T, V> r;
    if constexpr (V == 1) {
        r.v[0] = __ldg(p);
    } else if constexpr (std::is_same<T, double>::value && V == 2) {
        const double2 d = __ldg(reinterpret_cast<const double2*>(p));
        r.v[0] = d.x;
        r.v[1] = d.y;
    } else if constexpr (std::is_same<T, float>::value && V == 2) {
        const float2 d = __ldg(reinterpret_cast<const float2*>(p));
        r.v[0] = d.x;
        r.v[1] = d.y;
    } else {
        static_assert(std::is_same<T, float>::value && V == 4, "unsupported pack");
        const float4 d = __ldg(reinterpret_cast<const float4*>(p));
        r.v[0] = d.x;
        r.v[1] = d.y;
        r.v[2] = d.z;
        r.v[3] = d.w;
    }
    return r;
}

// L2 load (rows written by other SMs during this launch must not come from a stale L1 line).
template <typename T, int V>
__device__ __forceinline__ Pack<T, V> ld_l2(const T* p) {
    Pack<T, V> r;
    if constexpr (V == 1) {
        r.v[0] = __ldcg(p);
    } else if constexpr (std::is_same<T, double>::value && V == 2) {
        const double2 d = __ldcg(reinterpret_cast<const double2*>(p));
        r.v[0] = d.x;
        r.v[1] = d.y;
    } else if constexpr (std::is_same<T, float>::value && V == 2) {
        const float2 d = __ldcg(reinterpret_cast<const float2*>(p));
        r.v[0] = d.x;
        r.v[1] = d.y;
    } else {
        const float4 d = __ldcg(reinterpret_cast<const float4*>(p));
        r.v[0] = d.x;
        r.v[1] = d.y;
        r.v[2] = d.z;
        r.v[3] = d.w;
    }
    return r;
}

// Source-row load of the level walkers: the read-only path, or L2 only (CG) where rows read
// here may have been written by other SMs earlier in the same launch.
template <typename T, int V, bool CG>
__device__ __forceinline__ Pack<T, V> ld_src(const T* p) {
    if constexpr (CG) return ld_l2<T, V>(p);
    else return ld_ro<T, V>(p);
}

template <typename T, int V>
__device__ __forceinline__ void st_pack(T* p, const Pack<T, V>& x) {
    *reinterpret_cast<Pack<T, V>*>(p) = x;
}

__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

// ---------------------------------------------------------------------------------------
// Kernel parameters
// ---------------------------------------------------------------------------------------
struct LevelArgs {
    int64_t row_begin;
    int64_t num_rows;
    const int32_t* row_ptr;
    const uint32_t* entries;
    const int32_t* heavy_rows;
    const int32_t* row_ids;
    int64_t num_heavy;
    int32_t heavy_threshold;
    int32_t list_align;
    int32_t use_miss;
    void* state;
    int64_t ld_state;
    const void* x;
    int64_t ld_x;
    const void* miss;
    int64_t ld_miss;
    const void* init_vector;
    const void* init_matrix;
    int64_t ld_init;
    const int32_t* node_perm;
    const void* xtx_node;
    int64_t k;
    int32_t log2g;
    int32_t* err;
    int64_t lim_state;
    int64_t lim_x;
    int64_t lim_miss;
    int32_t log2s;  // narrow rows split over 2^log2s lane groups (default mode, variant 6)
    int32_t num_slot_buckets;  // > 0: narrow lists located from the slot table, not row_ptr
    int32_t slot_width[GRG_B200_MAX_SLOT_BUCKETS];
    int64_t slot_pos[GRG_B200_MAX_SLOT_BUCKETS];
    int64_t slot_entry[GRG_B200_MAX_SLOT_BUCKETS];
    // mixed storage only: the 16-bit planes of state, x and miss (x/miss hold encoded copies)
    void* state_lo;
    const void* x_lo;
    const void* miss_lo;
    int32_t up;  // an up level: its lists name state rows (and null padding) only
    int64_t short_rows;  // entry kernels: the last short_rows narrow positions take one entry slot
};

enum DeviceError : int32_t {
    kErrStateId = 1,
    kErrInputId = 2,
    kErrMissId = 3,
    kErrPerm = 4,
    kErrSelector = 5,
    kErrWaitTimeout = 6,  // dataflow: a source row never became ready within the spin limit
};

__device__ __forceinline__ void report(int32_t* err, int32_t code) {
    if (err) atomicCAS(err, 0, code);
}

// Programmatic dependent launch: a kernel launched with it may start while the previous
// kernel of the stream is finishing; it reads only static data (level lists) until
// pdl_wait(), which returns once the previous grid has completed and its writes are visible
// (immediately when the launch did not use the attribute).  pdl_trigger() lets the next
// kernel launch once every CTA of this grid has started.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" :::); }

template <typename T, int V, int INIT>
__device__ __forceinline__ Pack<T, V> init_value(const LevelArgs& a, int64_t row, int64_t c) {
    if constexpr (INIT == GRG_B200_INIT_VECTOR) {
        return ld_ro<T, V>(static_cast<const T*>(a.init_vector) + c);
    } else if constexpr (INIT == GRG_B200_INIT_XTX) {
        return splat<T, V>(__ldg(static_cast<const T*>(a.xtx_node) + row));
    } else if constexpr (INIT == GRG_B200_INIT_MATRIX) {
        const int64_t orig = __ldg(a.node_perm + row);
        if (a.err && (orig < 0 || orig >= a.lim_state)) {
            report(a.err, kErrPerm);
            return zero_pack<T, V>();
        }
        return ld_ro<T, V>(static_cast<const T*>(a.init_matrix) + orig * a.ld_init + c);
    } else {
        return zero_pack<T, V>();
    }
}

// Address of the row named by a coded entry; nullptr when the entry is skipped.
template <typename T>
__device__ __forceinline__ const T* entry_row(const LevelArgs& a, uint32_t code) {
    const uint32_t src = (code >> GRG_B200_SRC_SHIFT) & GRG_B200_SRC_MASK;
    const int64_t id = code & GRG_B200_ID_MASK;
    if (src == GRG_B200_SRC_STATE) {
        if (a.err && id >= a.lim_state) {
            report(a.err, kErrStateId);
            return nullptr;
        }
        return static_cast<const T*>(a.state) + id * a.ld_state;
    }
    if (src == GRG_B200_SRC_INPUT) {
        if (a.err && id >= a.lim_x) {
            report(a.err, kErrInputId);
            return nullptr;
        }
        return static_cast<const T*>(a.x) + id * a.ld_x;
    }
    if (src != GRG_B200_SRC_MISS || !a.use_miss) return nullptr;  // null padding, or miss rows off
    if (a.err && id >= a.lim_miss) {
        report(a.err, kErrMissId);
        return nullptr;
    }
    return static_cast<const T*>(a.miss) + id * a.ld_miss;
}

// ---------------------------------------------------------------------------------------
// Level kernels
// ---------------------------------------------------------------------------------------
constexpr int kNarrowThreads = 256;
constexpr int kNarrowWarps = kNarrowThreads / 32;
constexpr int kStageCap = 1024;  // gather-list entries staged in shared memory per warp
constexpr unsigned kFullMask = 0xffffffffu;

__device__ __forceinline__ int64_t level_row(const LevelArgs& a, int64_t pos) {
    return a.row_begin + (a.row_ids ? static_cast<int64_t>(__ldg(a.row_ids + pos)) : pos);
}

// Narrow rows.  A warp owns 32/G consecutive processing positions; lane group g (G lanes)
// owns position g and columns [lane*V, lane*V + V) (+ multiples of G*V).  The warp first
// copies the gather-list span of its positions into shared memory with coalesced loads;
// each lane then fetches U rows at a time (independent loads) and adds them in list order,
// restarting the partial sum at every segment start.
//
// Variants (``narrow_variant``): U = rows fetched per round, STAGE = shared-memory staging.
template <typename T, int V, int INIT, int U, bool STAGE, int MIN_BLOCKS = 1>
__global__ void __launch_bounds__(kNarrowThreads, MIN_BLOCKS) level_narrow_kernel(LevelArgs a) {
    __shared__ uint32_t stage[kNarrowWarps][STAGE ? kStageCap : 1];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int rpw_log = 5 - a.log2g;  // positions per warp = 32 >> log2g
    const int64_t narrow = a.num_rows - a.num_heavy;  // heavy positions form the suffix
    const int64_t pos0 = (static_cast<int64_t>(blockIdx.x) * kNarrowWarps + warp) << rpw_log;
    if (pos0 >= narrow) return;  // uniform across the warp
    const int here = static_cast<int>(narrow - pos0 < (int64_t(1) << rpw_log) ? narrow - pos0 : (int64_t(1) << rpw_log));
    // Lane l < here holds the list bounds of position pos0 + l (a full warp of single-lane
    // rows needs 33 offsets, so each lane loads both ends of its own position).
    int32_t lo = 0, hi = 0;
    if (lane < here) {
        lo = __ldg(a.row_ptr + pos0 + lane);
        hi = __ldg(a.row_ptr + pos0 + lane + 1);
    }
    const int32_t span_begin = __shfl_sync(kFullMask, lo, 0);
    const int32_t span = __shfl_sync(kFullMask, hi, here - 1) - span_begin;
    const int my = lane >> a.log2g;
    const int owner = my < here ? my : 0;
    const int32_t e0 = __shfl_sync(kFullMask, lo, owner);
    const int32_t e1 = __shfl_sync(kFullMask, hi, owner);
    const bool staged = STAGE && span <= kStageCap;
    if (staged) {
        for (int j = lane; j < span; j += 32) stage[warp][j] = __ldg(a.entries + span_begin + j);
    }
    __syncwarp();
    if (my >= here) return;
    const int glane = lane & ((1 << a.log2g) - 1);
    const int64_t row = level_row(a, pos0 + my);
    T* state = static_cast<T*>(a.state);
    const uint32_t* stage_w = stage[warp];
    const int64_t step = static_cast<int64_t>(V) << a.log2g;
    for (int64_t c = static_cast<int64_t>(glane) * V; c < a.k; c += step) {
        Pack<T, V> acc = init_value<T, V, INIT>(a, row, c);
        Pack<T, V> seg = zero_pack<T, V>();
        for (int32_t e = e0; e < e1; e += U) {
            uint32_t code[U];
            Pack<T, V> val[U];
            bool valid[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int32_t eu = e + u;
                code[u] = eu >= e1 ? 0u : (staged ? stage_w[eu - span_begin] : __ldg(a.entries + eu));
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const T* src = (e + u < e1) ? entry_row<T>(a, code[u]) : nullptr;
                valid[u] = src != nullptr;
                val[u] = valid[u] ? ld_ro<T, V>(src + c) : zero_pack<T, V>();
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (code[u] & GRG_B200_SEG_START) {
                    add_into(acc, seg);
                    seg = zero_pack<T, V>();
                }
                if (valid[u]) add_into(seg, val[u]);
            }
        }
        add_into(acc, seg);
        st_pack(state + row * a.ld_state + c, acc);
    }
}

// cp.async helpers: global -> shared copies that hold no registers while in flight.
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
    const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    if constexpr (BYTES == 16) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(gmem) : "memory");
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(dst), "l"(gmem), "n"(BYTES) : "memory");
    }
}

__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

constexpr int kAsyncWarps = 4;
constexpr int kAsyncThreads = kAsyncWarps * 32;
constexpr int kAsyncValBytes = 8192;  // gathered row segments per warp and round
constexpr int kAsyncCodeCap = 512;    // list entries per warp and round

// Narrow rows, asynchronous gathers (narrow_variant 4).  Same ownership as
// level_narrow_kernel (a warp owns 32/G positions, lane group g owns position g).  Per round
// the warp copies up to `cap` list entries of its span into shared memory, issues one
// cp.async per (entry, lane) for the entry's row segment [c0 + lane*V, +V), waits once, and
// every lane group then adds its own row's entries from shared memory in list order.  All row
// fetches of a round are in flight at once without occupying registers.
template <typename T, int V, int INIT>
__global__ void __launch_bounds__(kAsyncThreads) level_async_kernel(LevelArgs a) {
    __shared__ __align__(16) unsigned char vals_raw[kAsyncWarps][kAsyncValBytes];
    __shared__ uint32_t codes_s[kAsyncWarps][kAsyncCodeCap];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int rpw_log = 5 - a.log2g;
    const int64_t narrow = a.num_rows - a.num_heavy;  // heavy positions form the suffix
    const int64_t pos0 = (static_cast<int64_t>(blockIdx.x) * kAsyncWarps + warp) << rpw_log;
    if (pos0 >= narrow) return;  // uniform across the warp
    const int here = static_cast<int>(narrow - pos0 < (int64_t(1) << rpw_log) ? narrow - pos0 : (int64_t(1) << rpw_log));
    int32_t lo = 0, hi = 0;
    if (lane < here) {
        lo = __ldg(a.row_ptr + pos0 + lane);
        hi = __ldg(a.row_ptr + pos0 + lane + 1);
    }
    const int32_t span_begin = __shfl_sync(kFullMask, lo, 0);
    const int32_t span_end = __shfl_sync(kFullMask, hi, here - 1);
    const int my = lane >> a.log2g;
    const int owner = my < here ? my : 0;
    const int32_t e0 = __shfl_sync(kFullMask, lo, owner);
    const int32_t e1 = __shfl_sync(kFullMask, hi, owner);
    const bool has_row = my < here;
    const int g_lanes = 1 << a.log2g;
    const int g = lane & (g_lanes - 1);
    const int64_t row = has_row ? level_row(a, pos0 + my) : 0;
    Pack<T, V>* vals = reinterpret_cast<Pack<T, V>*>(vals_raw[warp]);
    uint32_t* codes = codes_s[warp];
    const int per_entry = static_cast<int>(sizeof(T)) * V << a.log2g;
    const int cap = kAsyncValBytes / per_entry < kAsyncCodeCap ? kAsyncValBytes / per_entry : kAsyncCodeCap;
    T* state = static_cast<T*>(a.state);
    const int64_t cstep = static_cast<int64_t>(V) << a.log2g;
    for (int64_t c0 = 0; c0 < a.k; c0 += cstep) {
        const int64_t c = c0 + static_cast<int64_t>(g) * V;
        const bool live = has_row && c < a.k;
        Pack<T, V> acc = live ? init_value<T, V, INIT>(a, row, c) : zero_pack<T, V>();
        Pack<T, V> seg = zero_pack<T, V>();
        for (int32_t sub = span_begin; sub < span_end; sub += cap) {
            const int n = span_end - sub < cap ? span_end - sub : cap;
            for (int j = lane; j < n; j += 32) codes[j] = __ldg(a.entries + sub + j);
            __syncwarp();
            for (int q = lane; q < (n << a.log2g); q += 32) {
                const int j = q >> a.log2g;
                const int64_t cc = c0 + static_cast<int64_t>(q & (g_lanes - 1)) * V;
                const T* src = entry_row<T>(a, codes[j]);
                if (src && cc < a.k) cp_async<static_cast<int>(sizeof(T)) * V>(&vals[q], src + cc);
            }
            cp_async_wait_all();
            __syncwarp();
            if (live) {
                const int32_t lo_e = e0 > sub ? e0 : sub;
                const int32_t hi_e = e1 < sub + n ? e1 : sub + n;
                for (int32_t e = lo_e; e < hi_e; ++e) {
                    const uint32_t code = codes[e - sub];
                    if (code & GRG_B200_SEG_START) {
                        add_into(acc, seg);
                        seg = zero_pack<T, V>();
                    }
                    if (entry_row<T>(a, code)) add_into(seg, vals[((e - sub) << a.log2g) + g]);
                }
            }
            __syncwarp();
        }
        if (live) {
            add_into(acc, seg);
            st_pack(state + row * a.ld_state + c, acc);
        }
    }
}

// Narrow rows from padded lists (narrow_variant 6).  Same ownership as level_narrow_kernel; a
// lane reads its row's codes four at a time with one aligned 16-byte load and loads the next
// four while the current four rows are fetched, so each round waits on one memory latency.
// A narrow row's list: from the slot table when the level has one (no dependent load), else
// from row_ptr.
__device__ __forceinline__ void narrow_extent(const LevelArgs& a, int64_t pos, int32_t& e0, int32_t& e1) {
    if (a.num_slot_buckets > 0) {
        int b = 0;
#pragma unroll
        for (int i = 1; i < GRG_B200_MAX_SLOT_BUCKETS; ++i)
            if (i < a.num_slot_buckets && pos >= a.slot_pos[i]) b = i;
        const int32_t w = 4 * a.slot_width[b];
        e0 = static_cast<int32_t>(a.slot_entry[b] + (pos - a.slot_pos[b]) * w);
        e1 = e0 + w;
    } else {
        e0 = __ldg(a.row_ptr + pos);
        e1 = __ldg(a.row_ptr + pos + 1);
    }
}

template <typename T, int V, int INIT, int Q = 1, bool CG = false>
__device__ __forceinline__ void vec_rows(const LevelArgs& a, int64_t block) {
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int64_t narrow = a.num_rows - a.num_heavy;  // heavy positions form the suffix
    const int64_t pos = ((block * kNarrowWarps + warp) << (5 - a.log2g)) + (lane >> a.log2g);
    if (pos >= narrow) return;  // no warp-wide operations below
    int32_t e0, e1;
    narrow_extent(a, pos, e0, e1);
    const int glane = lane & ((1 << a.log2g) - 1);
    const int64_t row = level_row(a, pos);
    const uint4* codes4 = reinterpret_cast<const uint4*>(a.entries);
    const uint32_t null_code = GRG_B200_SRC_NULL << GRG_B200_SRC_SHIFT;
    const uint4 null4 = make_uint4(null_code, null_code, null_code, null_code);
    uint4 first[Q];  // the list is static: fetched before waiting for the previous level
#pragma unroll
    for (int j = 0; j < Q; ++j) first[j] = (e0 >> 2) + j < (e1 >> 2) ? __ldg(codes4 + (e0 >> 2) + j) : null4;
    pdl_wait();
    T* state = static_cast<T*>(a.state);
    const int64_t step = static_cast<int64_t>(V) << a.log2g;
    for (int64_t c = static_cast<int64_t>(glane) * V; c < a.k; c += step) {
        Pack<T, V> acc = init_value<T, V, INIT>(a, row, c);
        Pack<T, V> seg = zero_pack<T, V>();
        const int32_t q1 = e1 >> 2;
        int32_t q = e0 >> 2;
        uint4 cur[Q];
#pragma unroll
        for (int j = 0; j < Q; ++j) cur[j] = first[j];
        for (; q < q1; q += Q) {  // Q quads (4 * Q row fetches) in flight per round
            uint4 nxt[Q];
#pragma unroll
            for (int j = 0; j < Q; ++j) nxt[j] = q + Q + j < q1 ? __ldg(codes4 + q + Q + j) : null4;
            uint32_t code[4 * Q];
#pragma unroll
            for (int j = 0; j < Q; ++j) {
                code[4 * j] = cur[j].x;
                code[4 * j + 1] = cur[j].y;
                code[4 * j + 2] = cur[j].z;
                code[4 * j + 3] = cur[j].w;
            }
            Pack<T, V> val[4 * Q];
            bool valid[4 * Q];
#pragma unroll
            for (int u = 0; u < 4 * Q; ++u) {
                const T* src = entry_row<T>(a, code[u]);
                valid[u] = src != nullptr;
                val[u] = valid[u] ? ld_src<T, V, CG>(src + c) : zero_pack<T, V>();
            }
#pragma unroll
            for (int u = 0; u < 4 * Q; ++u) {
                if (code[u] & GRG_B200_SEG_START) {
                    add_into(acc, seg);
                    seg = zero_pack<T, V>();
                }
                if (valid[u]) add_into(seg, val[u]);
            }
#pragma unroll
            for (int j = 0; j < Q; ++j) cur[j] = nxt[j];
        }
        add_into(acc, seg);
        st_pack(state + row * a.ld_state + c, acc);
    }
}

template <typename T, int V>
__device__ __forceinline__ Pack<T, V> shfl_xor_pack(const Pack<T, V>& x, int off) {
    Pack<T, V> r;
#pragma unroll
    for (int i = 0; i < V; ++i) r.v[i] = __shfl_xor_sync(kFullMask, x.v[i], off);
    return r;
}

// Narrow rows of padded lists, each split over 2^log2s lane groups (default mode only): group
// j of a row takes quads j, j + 2^log2s, ... and the groups' sums are combined by an
// xor-shuffle butterfly in a fixed order, so a row waits on ~1/2^log2s of the memory round
// trips of vec_rows.  Used for levels whose rows are long but too few to fill the GPU.
template <typename T, int V, int INIT>
__device__ __forceinline__ void split_rows(const LevelArgs& a, int64_t block) {
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int lg = a.log2g + a.log2s;  // lanes per row
    const int64_t narrow = a.num_rows - a.num_heavy;
    const int64_t pos = ((block * kNarrowWarps + warp) << (5 - lg)) + (lane >> lg);
    const bool live = pos < narrow;  // dead lanes still join the shuffles
    int32_t e0 = 0, e1 = 0;
    int64_t row = 0;
    if (live) {
        e0 = __ldg(a.row_ptr + pos);
        e1 = __ldg(a.row_ptr + pos + 1);
        row = level_row(a, pos);
    }
    pdl_wait();
    const int glane = lane & ((1 << a.log2g) - 1);
    const int sub = (lane >> a.log2g) & ((1 << a.log2s) - 1);
    const uint4* codes4 = reinterpret_cast<const uint4*>(a.entries);
    T* state = static_cast<T*>(a.state);
    const int64_t step = static_cast<int64_t>(V) << a.log2g;
    for (int64_t c = static_cast<int64_t>(glane) * V; c < a.k; c += step) {  // same trip count in every lane
        Pack<T, V> part = zero_pack<T, V>();
        if (live) {
            for (int32_t q = (e0 >> 2) + sub; q < (e1 >> 2); q += 1 << a.log2s) {
                const uint4 cq = __ldg(codes4 + q);
                const uint32_t code[4] = {cq.x, cq.y, cq.z, cq.w};
                Pack<T, V> val[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const T* src = entry_row<T>(a, code[u]);
                    val[u] = src ? ld_ro<T, V>(src + c) : zero_pack<T, V>();
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) add_into(part, val[u]);
            }
        }
        for (int off = 1 << a.log2g; off < (1 << lg); off <<= 1) {
            const Pack<T, V> other = shfl_xor_pack(part, off);
            add_into(part, other);
        }
        if (live && sub == 0) {
            Pack<T, V> acc = init_value<T, V, INIT>(a, row, c);
            add_into(acc, part);
            st_pack(state + row * a.ld_state + c, acc);
        }
    }
}

// MB = CTAs per SM the register budget is sized for: 6 (narrow_variant 6, 40 registers), 5
// (narrow_variant 7, 48 registers: no spills, fewer warps) or 3 (narrow_variant 8, Q = 2: two
// quads, eight row fetches, in flight per round).
template <typename T, int V, int INIT, int MB, int Q = 1>
__global__ void __launch_bounds__(kNarrowThreads, MB) level_vec_kernel(LevelArgs a) {
    pdl_trigger();
    vec_rows<T, V, INIT, Q>(a, blockIdx.x);
}

constexpr int kWarpRowThreads = 256;

// Heavy rows, one warp each (heavy_variant 1, default mode only).  Lane group g of 32/G
// groups takes every (32/G)-th 4-entry quad of the row's list (or every (32/G)-th entry for
// unpadded lists) and fetches its rows independently; the groups' partial sums are combined
// by an xor-shuffle butterfly in a fixed order, so the result is deterministic (and exact for
// integer data), and group 0 adds the init value and stores the row.  Compared with a CTA per
// row this keeps eight heavy rows per CTA and needs no shared memory or block barriers.
template <typename T, int V, int INIT, int WPC = kWarpRowThreads / 32, bool CG = false>
__device__ __forceinline__ void warp_heavy_rows(const LevelArgs& a, int64_t block) {
    const int64_t w = block * WPC + (threadIdx.x >> 5);
    if (w >= a.num_heavy) return;  // warp-uniform
    const int lane32 = threadIdx.x & 31;
    const int64_t pos = __ldg(a.heavy_rows + w);
    const int32_t e0 = __ldg(a.row_ptr + pos);
    const int32_t e1 = __ldg(a.row_ptr + pos + 1);
    const int64_t row = level_row(a, pos);
    pdl_wait();
    const int g_lanes = 1 << a.log2g;
    const int groups = 32 >> a.log2g;
    const int glane = lane32 & (g_lanes - 1);
    const int grp = lane32 >> a.log2g;
    T* state = static_cast<T*>(a.state);
    const int64_t step = static_cast<int64_t>(V) << a.log2g;
    for (int64_t base = 0; base < a.k; base += step) {  // uniform trip count across the warp
        const int64_t c = base + static_cast<int64_t>(glane) * V;
        const bool active = c < a.k;
        Pack<T, V> part = zero_pack<T, V>();
        if (active) {
            if (a.list_align == 4) {
                // this group's quads are q0, q0 + groups, ...: the next one's codes load while the
                // current four rows are fetched, so a round waits on one memory latency
                const uint4* codes4 = reinterpret_cast<const uint4*>(a.entries);
                const uint32_t null_code = GRG_B200_SRC_NULL << GRG_B200_SRC_SHIFT;
                const uint4 null4 = make_uint4(null_code, null_code, null_code, null_code);
                const int32_t q1 = e1 >> 2;
                int32_t q = (e0 >> 2) + grp;
                uint4 cur = q < q1 ? __ldg(codes4 + q) : null4;
                for (; q < q1; q += groups) {
                    const uint4 nxt = q + groups < q1 ? __ldg(codes4 + q + groups) : null4;
                    const uint32_t code[4] = {cur.x, cur.y, cur.z, cur.w};
                    Pack<T, V> val[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const T* src = entry_row<T>(a, code[u]);
                        val[u] = src ? ld_src<T, V, CG>(src + c) : zero_pack<T, V>();
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) add_into(part, val[u]);
                    cur = nxt;
                }
            } else {
                constexpr int UW = 4;
                for (int32_t j = e0 + grp; j < e1; j += groups * UW) {
                    Pack<T, V> val[UW];
#pragma unroll
                    for (int u = 0; u < UW; ++u) {
                        const int32_t jj = j + u * groups;
                        const T* src = jj < e1 ? entry_row<T>(a, __ldg(a.entries + jj)) : nullptr;
                        val[u] = src ? ld_src<T, V, CG>(src + c) : zero_pack<T, V>();
                    }
#pragma unroll
                    for (int u = 0; u < UW; ++u) add_into(part, val[u]);
                }
            }
        }
        for (int off = 16; off >= g_lanes; off >>= 1) {
            const Pack<T, V> other = shfl_xor_pack(part, off);
            add_into(part, other);
        }
        if (grp == 0 && active) {
            Pack<T, V> acc = init_value<T, V, INIT>(a, row, c);
            add_into(acc, part);
            st_pack(state + row * a.ld_state + c, acc);
        }
    }
}

// WPC = heavy rows (warps) per CTA: 8, or 32 for heavy_variant 3 (consecutive rows, which
// share sources in locality order, then share an SM's L1).
template <typename T, int V, int INIT, int WPC = kWarpRowThreads / 32>
__global__ void __launch_bounds__(WPC * 32) level_warp_kernel(LevelArgs a) {
    pdl_trigger();
    warp_heavy_rows<T, V, INIT, WPC>(a, blockIdx.x);
}

// One launch for a whole level (heavy_variant 2): the first ceil(num_heavy / 8) CTAs take the
// heavy rows one warp each, so the longest lists start first, and the remaining CTAs take the
// narrow rows as level_vec_kernel does.  The two kinds of rows are disjoint and read only
// lower levels, so nothing orders them; this saves the second launch of a level and lets the
// heavy rows overlap the narrow ones.
template <typename T, int V, int INIT, bool SPLIT, int MB, int Q = 1>
__global__ void __launch_bounds__(kNarrowThreads, MB) level_fused_kernel(LevelArgs a, int64_t heavy_blocks) {
    static_assert(kNarrowThreads == kWarpRowThreads, "both row kinds use the same CTA shape");
    pdl_trigger();
    if (static_cast<int64_t>(blockIdx.x) < heavy_blocks) warp_heavy_rows<T, V, INIT>(a, blockIdx.x);
    else if constexpr (SPLIT) split_rows<T, V, INIT>(a, static_cast<int64_t>(blockIdx.x) - heavy_blocks);
    else vec_rows<T, V, INIT, Q>(a, static_cast<int64_t>(blockIdx.x) - heavy_blocks);
}

// Lean row walks (narrow_variant 11 and 12): the same rows and the same arithmetic as
// vec_rows / warp_heavy_rows, for the common launch: no bounds checks (the launch has no error
// word), source rows addressed with one 32 x 32 -> 64-bit multiply (row ids and leading
// dimensions are below 2^32), and for up levels a state-only decode (up lists name state rows
// and null padding only; input rows reach up through the level-0 seed).  SEG = true keeps a
// fresh partial sum per segment, so results are bit-identical to vec_rows; SEG = false adds a
// row's entries left to right into one sum (default mode only: integer-valued inputs stay
// exact, real-valued ones differ from the reference by reassociation).
template <typename T, bool UPONLY>
__device__ __forceinline__ const T* lean_source(const LevelArgs& a, uint32_t code, bool& ok) {
    const uint32_t id = code & GRG_B200_ID_MASK;
    const uint32_t src = (code >> GRG_B200_SRC_SHIFT) & GRG_B200_SRC_MASK;
    if constexpr (UPONLY) {
        ok = src == GRG_B200_SRC_STATE;
        return static_cast<const T*>(a.state) + static_cast<size_t>(id) * static_cast<uint32_t>(a.ld_state);
    } else {
        ok = src == GRG_B200_SRC_STATE || src == GRG_B200_SRC_INPUT || (src == GRG_B200_SRC_MISS && a.use_miss);
        const T* base = src == GRG_B200_SRC_STATE ? static_cast<const T*>(a.state)
                                                   : (src == GRG_B200_SRC_INPUT ? static_cast<const T*>(a.x) : static_cast<const T*>(a.miss));
        const uint32_t ld = static_cast<uint32_t>(src == GRG_B200_SRC_STATE ? a.ld_state : (src == GRG_B200_SRC_INPUT ? a.ld_x : a.ld_miss));
        return base + static_cast<size_t>(id) * ld;
    }
}

template <typename T, int V, int INIT, bool SEG, bool UPONLY, int NW = kNarrowWarps>
__device__ __forceinline__ void lean_rows(const LevelArgs& a, int64_t block) {
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int64_t narrow = a.num_rows - a.num_heavy;  // heavy positions form the suffix
    const int64_t pos = ((block * NW + warp) << (5 - a.log2g)) + (lane >> a.log2g);
    if (pos >= narrow) return;  // no warp-wide operations below
    const int32_t q0 = __ldg(a.row_ptr + pos) >> 2;
    const int32_t q1 = __ldg(a.row_ptr + pos + 1) >> 2;
    const int glane = lane & ((1 << a.log2g) - 1);
    const int64_t row = level_row(a, pos);
    const uint4* codes4 = reinterpret_cast<const uint4*>(a.entries);
    const uint32_t null_code = GRG_B200_SRC_NULL << GRG_B200_SRC_SHIFT;
    const uint4 null4 = make_uint4(null_code, null_code, null_code, null_code);
    const uint4 first = q0 < q1 ? __ldg(codes4 + q0) : null4;  // static list: before the wait
    pdl_wait();
    T* state = static_cast<T*>(a.state);
    const int step = V << a.log2g;
    const int k = static_cast<int>(a.k);
    for (int c = glane * V; c < k; c += step) {
        Pack<T, V> acc = init_value<T, V, INIT>(a, row, c);
        Pack<T, V> seg = zero_pack<T, V>();
        uint4 cur = first;
        for (int32_t q = q0; q < q1; ++q) {
            const uint4 nxt = q + 1 < q1 ? __ldg(codes4 + q + 1) : null4;
            const uint32_t code[4] = {cur.x, cur.y, cur.z, cur.w};
            Pack<T, V> val[4];
            bool ok[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const T* p = lean_source<T, UPONLY>(a, code[u], ok[u]);
                val[u] = ok[u] ? ld_ro<T, V>(p + c) : zero_pack<T, V>();
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if constexpr (SEG) {
                    if (code[u] & GRG_B200_SEG_START) {
                        add_into(acc, seg);
                        seg = zero_pack<T, V>();
                    }
                    if (ok[u]) add_into(seg, val[u]);
                } else {
                    if (ok[u]) add_into(acc, val[u]);
                }
            }
            cur = nxt;
        }
        if constexpr (SEG) add_into(acc, seg);
        st_pack(state + row * a.ld_state + c, acc);
    }
}

// Heavy rows, one warp each, as warp_heavy_rows (padded lists) with the lean decode.
template <typename T, int V, int INIT, bool UPONLY, int WPC = kWarpRowThreads / 32>
__device__ __forceinline__ void lean_heavy_rows(const LevelArgs& a, int64_t block) {
    const int64_t w = block * WPC + (threadIdx.x >> 5);
    if (w >= a.num_heavy) return;  // warp-uniform
    const int lane32 = threadIdx.x & 31;
    const int64_t pos = __ldg(a.heavy_rows + w);
    const int32_t q1 = __ldg(a.row_ptr + pos + 1) >> 2;
    const int32_t qs = __ldg(a.row_ptr + pos) >> 2;
    const int64_t row = level_row(a, pos);
    pdl_wait();
    const int g_lanes = 1 << a.log2g;
    const int groups = 32 >> a.log2g;
    const int glane = lane32 & (g_lanes - 1);
    const int grp = lane32 >> a.log2g;
    T* state = static_cast<T*>(a.state);
    const uint4* codes4 = reinterpret_cast<const uint4*>(a.entries);
    const uint32_t null_code = GRG_B200_SRC_NULL << GRG_B200_SRC_SHIFT;
    const uint4 null4 = make_uint4(null_code, null_code, null_code, null_code);
    const int step = V << a.log2g;
    const int k = static_cast<int>(a.k);
    for (int base = 0; base < k; base += step) {  // uniform trip count across the warp
        const int c = base + glane * V;
        const bool active = c < k;
        Pack<T, V> part = zero_pack<T, V>();
        if (active) {
            int32_t q = qs + grp;
            uint4 cur = q < q1 ? __ldg(codes4 + q) : null4;
            for (; q < q1; q += groups) {
                const uint4 nxt = q + groups < q1 ? __ldg(codes4 + q + groups) : null4;
                const uint32_t code[4] = {cur.x, cur.y, cur.z, cur.w};
                Pack<T, V> val[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    bool ok;
                    const T* p = lean_source<T, UPONLY>(a, code[u], ok);
                    val[u] = ok ? ld_ro<T, V>(p + c) : zero_pack<T, V>();
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) add_into(part, val[u]);
                cur = nxt;
            }
        }
        for (int off = 16; off >= g_lanes; off >>= 1) {
            const Pack<T, V> other = shfl_xor_pack(part, off);
            add_into(part, other);
        }
        if (grp == 0 && active) {
            Pack<T, V> acc = init_value<T, V, INIT>(a, row, c);
            add_into(acc, part);
            st_pack(state + row * a.ld_state + c, acc);
        }
    }
}

// 32-byte vector loads and stores (sm_100): one chunk of 4 doubles or 8 floats.
template <typename T>
struct Chunk32 {
    static constexpr int C = 32 / static_cast<int>(sizeof(T));
    using type = Pack<T, C>;
};

template <typename T>
__device__ __forceinline__ typename Chunk32<T>::type ld_chunk(const T* p) {
    typename Chunk32<T>::type r;
    if constexpr (std::is_same<T, double>::value) {
        asm volatile("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
                     : "=d"(r.v[0]), "=d"(r.v[1]), "=d"(r.v[2]), "=d"(r.v[3]) : "l"(p));
    } else {
        asm volatile("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                     : "=f"(r.v[0]), "=f"(r.v[1]), "=f"(r.v[2]), "=f"(r.v[3]), "=f"(r.v[4]), "=f"(r.v[5]), "=f"(r.v[6]), "=f"(r.v[7])
                     : "l"(p));
    }
    return r;
}

// One chunk lane's CW columns: a 32-byte load when CW fills a chunk, else the shape's vector
// load (k below a chunk: CW = k, one chunk lane per row).
template <typename T, int CW>
__device__ __forceinline__ Pack<T, CW> ld_cols(const T* p) {
    if constexpr (CW == Chunk32<T>::C) return ld_chunk<T>(p);
    else return ld_ro<T, CW>(p);
}

// Narrow rows, entry-parallel (narrow_variant 13, default mode only).  A row's lane group of G
// lanes is W chunk lanes x 2 entry slots (W = k / CW): lane (e, w) adds chunk w of entries e and
// e + 2 of every 4-entry quad, so each code is decoded by W lanes instead of G and a row fetch
// is one load per chunk.  CW is a 32-byte chunk's columns, or, when k is a single vector of the
// shape (k below a chunk), k itself (W = 1).  The two slots' sums are added by one shuffle and
// the slot-0 lanes store.  The order of additions differs from the reference's (exact for
// integer-valued inputs, reassociation otherwise).  log2w = log2(W), G = 2W = 2^lg.
template <typename T, int INIT, bool UPONLY, int CW, int NW = kNarrowWarps>
__device__ __forceinline__ void entry_rows(const LevelArgs& a, int64_t block) {
    using Ch = Pack<T, CW>;
    constexpr int C = CW;  // columns per chunk lane
    const int lg = a.log2g + (CW == Chunk32<T>::C ? 0 : 1);  // log2 of the 2W lanes of a row
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int64_t narrow = a.num_rows - a.num_heavy - a.short_rows;  // the short rows follow
    const int64_t pos = ((block * NW + warp) << (5 - lg)) + (lane >> lg);
    const bool live = pos < narrow;  // dead lanes still join the shuffle
    const int glane = lane & ((1 << lg) - 1);
    const int log2w = lg - 1;
    const int w = glane & ((1 << log2w) - 1);
    const int e = glane >> log2w;  // entry slot 0 or 1
    int32_t q0 = 0, q1 = 0;
    int64_t row = 0;
    const uint4* codes4 = reinterpret_cast<const uint4*>(a.entries);
    const uint32_t null_code = GRG_B200_SRC_NULL << GRG_B200_SRC_SHIFT;
    const uint4 null4 = make_uint4(null_code, null_code, null_code, null_code);
    uint4 cur = null4;
    if (live) {
        q0 = __ldg(a.row_ptr + pos) >> 2;
        q1 = __ldg(a.row_ptr + pos + 1) >> 2;
        row = level_row(a, pos);
        if (q0 < q1) cur = __ldg(codes4 + q0);  // static list: before the wait
    }
    pdl_wait();
    const int c = w * C;
    Ch acc = zero_pack<T, C>();
    for (int32_t q = q0; q < q1; ++q) {
        const uint4 nxt = q + 1 < q1 ? __ldg(codes4 + q + 1) : null4;
        const uint32_t c0 = e == 0 ? cur.x : cur.y;  // entries e and e + 2 of the quad
        const uint32_t c1 = e == 0 ? cur.z : cur.w;
        bool ok0, ok1;
        const T* p0 = lean_source<T, UPONLY>(a, c0, ok0);
        const T* p1 = lean_source<T, UPONLY>(a, c1, ok1);
        const Ch v0 = ok0 ? ld_cols<T, CW>(p0 + c) : zero_pack<T, C>();
        const Ch v1 = ok1 ? ld_cols<T, CW>(p1 + c) : zero_pack<T, C>();
        add_into(acc, v0);
        add_into(acc, v1);
        cur = nxt;
    }
    const Ch other = shfl_xor_pack(acc, 1 << log2w);
    if (live && e == 0) {
        Ch out = init_value<T, C, INIT>(a, row, c);
        add_into(out, acc);
        add_into(out, other);
        st_pack(static_cast<T*>(a.state) + row * a.ld_state + c, out);
    }
}

// As entry_rows, with the codes of the row's first kPreQuads quads loaded before the wait
// (narrow_variant 14): a lane keeps its two codes of each (8 registers), so rows of up to
// 4 * kPreQuads entries walk their rounds without a code load on the critical path, and the
// loads overlap the previous level under programmatic dependent launch.  Longer rows load the
// rest one round ahead, as entry_rows does.
constexpr int kPreQuads = 4;

template <typename T, int INIT, bool UPONLY, int CW, int NW = kNarrowWarps>
__device__ __forceinline__ void entry_rows_pre(const LevelArgs& a, int64_t block) {
    using Ch = Pack<T, CW>;
    constexpr int C = CW;  // columns per chunk lane
    const int lg = a.log2g + (CW == Chunk32<T>::C ? 0 : 1);  // log2 of the 2W lanes of a row
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int64_t narrow = a.num_rows - a.num_heavy - a.short_rows;  // the short rows follow
    const int64_t pos = ((block * NW + warp) << (5 - lg)) + (lane >> lg);
    const bool live = pos < narrow;  // dead lanes still join the shuffle
    const int glane = lane & ((1 << lg) - 1);
    const int log2w = lg - 1;
    const int w = glane & ((1 << log2w) - 1);
    const int e = glane >> log2w;  // entry slot 0 or 1
    int32_t q0 = 0, q1 = 0;
    int64_t row = 0;
    const uint4* codes4 = reinterpret_cast<const uint4*>(a.entries);
    const uint32_t null_code = GRG_B200_SRC_NULL << GRG_B200_SRC_SHIFT;
    uint32_t pre0[kPreQuads], pre1[kPreQuads];  // this lane's entries e and e + 2 of the first quads
#pragma unroll
    for (int j = 0; j < kPreQuads; ++j) pre0[j] = pre1[j] = null_code;
    if (live) {
        q0 = __ldg(a.row_ptr + pos) >> 2;
        q1 = __ldg(a.row_ptr + pos + 1) >> 2;
        row = level_row(a, pos);
#pragma unroll
        for (int j = 0; j < kPreQuads; ++j) {
            if (q0 + j < q1) {  // static list: before the wait
                const uint4 cq = __ldg(codes4 + q0 + j);
                pre0[j] = e == 0 ? cq.x : cq.y;
                pre1[j] = e == 0 ? cq.z : cq.w;
            }
        }
    }
    pdl_wait();
    const int c = w * C;
    Ch acc = zero_pack<T, C>();
#pragma unroll
    for (int j = 0; j < kPreQuads; ++j) {
        if (q0 + j < q1) {
            bool ok0, ok1;
            const T* p0 = lean_source<T, UPONLY>(a, pre0[j], ok0);
            const T* p1 = lean_source<T, UPONLY>(a, pre1[j], ok1);
            const Ch v0 = ok0 ? ld_cols<T, CW>(p0 + c) : zero_pack<T, C>();
            const Ch v1 = ok1 ? ld_cols<T, CW>(p1 + c) : zero_pack<T, C>();
            add_into(acc, v0);
            add_into(acc, v1);
        }
    }
    if (q0 + kPreQuads < q1) {
        const uint4 null4 = make_uint4(null_code, null_code, null_code, null_code);
        uint4 cur = __ldg(codes4 + q0 + kPreQuads);
        for (int32_t q = q0 + kPreQuads; q < q1; ++q) {
            const uint4 nxt = q + 1 < q1 ? __ldg(codes4 + q + 1) : null4;
            const uint32_t c0 = e == 0 ? cur.x : cur.y;
            const uint32_t c1 = e == 0 ? cur.z : cur.w;
            bool ok0, ok1;
            const T* p0 = lean_source<T, UPONLY>(a, c0, ok0);
            const T* p1 = lean_source<T, UPONLY>(a, c1, ok1);
            const Ch v0 = ok0 ? ld_cols<T, CW>(p0 + c) : zero_pack<T, C>();
            const Ch v1 = ok1 ? ld_cols<T, CW>(p1 + c) : zero_pack<T, C>();
            add_into(acc, v0);
            add_into(acc, v1);
            cur = nxt;
        }
    }
    const Ch other = shfl_xor_pack(acc, 1 << log2w);
    if (live && e == 0) {
        Ch out = init_value<T, C, INIT>(a, row, c);
        add_into(out, acc);
        add_into(out, other);
        st_pack(static_cast<T*>(a.state) + row * a.ld_state + c, out);
    }
}

// The short narrow rows of the entry kernels: the last short_rows narrow positions, which hold
// at most one quad each, walked with one entry slot.  A row's W chunk lanes each add their
// 32-byte chunk of all the row's entries, left to right, so a warp covers 32 / W rows, twice as
// many as entry_rows, and a level of short rows needs half the CTAs.  The codes load before the
// wait; a longer list is still summed in full (one quad ahead, as entry_rows).
template <typename T, int INIT, bool UPONLY, int CW, int NW = kNarrowWarps>
__device__ __forceinline__ void entry_short_rows(const LevelArgs& a, int64_t block) {
    using Ch = Pack<T, CW>;
    constexpr int C = CW;  // columns per chunk lane
    const int lg = a.log2g + (CW == Chunk32<T>::C ? 0 : 1);  // log2 of the 2W lanes of a row
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int log2w = lg - 1;
    const int64_t narrow = a.num_rows - a.num_heavy;
    const int64_t pos = narrow - a.short_rows + ((block * NW + warp) << (5 - log2w)) + (lane >> log2w);
    const bool live = pos < narrow;
    const int w = lane & ((1 << log2w) - 1);
    int32_t q0 = 0, q1 = 0;
    int64_t row = 0;
    const uint4* codes4 = reinterpret_cast<const uint4*>(a.entries);
    const uint32_t null_code = GRG_B200_SRC_NULL << GRG_B200_SRC_SHIFT;
    const uint4 null4 = make_uint4(null_code, null_code, null_code, null_code);
    uint4 cur = null4;
    if (live) {
        q0 = __ldg(a.row_ptr + pos) >> 2;
        q1 = __ldg(a.row_ptr + pos + 1) >> 2;
        row = level_row(a, pos);
        if (q0 < q1) cur = __ldg(codes4 + q0);  // static list: before the wait
    }
    pdl_wait();
    if (!live) return;  // no shuffles below
    const int c = w * C;
    Ch acc = zero_pack<T, C>();
    for (int32_t q = q0; q < q1; ++q) {
        const uint4 nxt = q + 1 < q1 ? __ldg(codes4 + q + 1) : null4;
        const uint32_t code[4] = {cur.x, cur.y, cur.z, cur.w};
#pragma unroll
        for (int u = 0; u < 4; u += 2) {  // two fetches in flight, as in the two-slot walk
            bool ok0, ok1;
            const T* p0 = lean_source<T, UPONLY>(a, code[u], ok0);
            const T* p1 = lean_source<T, UPONLY>(a, code[u + 1], ok1);
            const Ch v0 = ok0 ? ld_cols<T, CW>(p0 + c) : zero_pack<T, C>();
            const Ch v1 = ok1 ? ld_cols<T, CW>(p1 + c) : zero_pack<T, C>();
            add_into(acc, v0);
            add_into(acc, v1);
        }
        cur = nxt;
    }
    Ch out = init_value<T, C, INIT>(a, row, c);
    add_into(out, acc);
    st_pack(static_cast<T*>(a.state) + row * a.ld_state + c, out);
}

// narrow_variant 14: CTAs [0, heavy_blocks) take the heavy rows (lean walk), the next
// long_blocks the two-slot narrow rows, the rest the short rows.
// NW warps per CTA: 8 (narrow_variant 14), 4 (15) or 2 (16): finer-grained CTAs at the same 40
// warps per SM.
template <typename T, int INIT, bool UPONLY, int CW, int NW = kNarrowWarps>
__global__ void __launch_bounds__(32 * NW, 40 / NW) level_entry_pre_kernel(LevelArgs a, int64_t heavy_blocks, int64_t long_blocks) {
    pdl_trigger();
    const int64_t b = blockIdx.x;
    if (b < heavy_blocks) lean_heavy_rows<T, (CW == Chunk32<T>::C ? CW / 2 : CW), INIT, UPONLY, NW>(a, b);
    else if (b < heavy_blocks + long_blocks) entry_rows_pre<T, INIT, UPONLY, CW, NW>(a, b - heavy_blocks);
    else entry_short_rows<T, INIT, UPONLY, CW, NW>(a, b - heavy_blocks - long_blocks);
}

// narrow_variant 13: as 14 with entry_rows for the two-slot narrow rows.
template <typename T, int INIT, bool UPONLY, int CW>
__global__ void __launch_bounds__(kNarrowThreads, 5) level_entry_kernel(LevelArgs a, int64_t heavy_blocks, int64_t long_blocks) {
    pdl_trigger();
    const int64_t b = blockIdx.x;
    if (b < heavy_blocks) lean_heavy_rows<T, (CW == Chunk32<T>::C ? CW / 2 : CW), INIT, UPONLY>(a, b);
    else if (b < heavy_blocks + long_blocks) entry_rows<T, INIT, UPONLY, CW>(a, b - heavy_blocks);
    else entry_short_rows<T, INIT, UPONLY, CW>(a, b - heavy_blocks - long_blocks);
}

// narrow_variant 11 (SEG) / 12: heavy rows first, one warp each, then the narrow rows, as
// level_fused_kernel; MB = 5 CTAs per SM.
// NW warps per CTA: 8, or 4 where variants 15 and 16 fall back to 12.
template <typename T, int V, int INIT, bool SEG, bool UPONLY, int NW = kNarrowWarps>
__global__ void __launch_bounds__(32 * NW, 40 / NW) level_lean_kernel(LevelArgs a, int64_t heavy_blocks) {
    pdl_trigger();
    if (static_cast<int64_t>(blockIdx.x) < heavy_blocks) lean_heavy_rows<T, V, INIT, UPONLY, NW>(a, blockIdx.x);
    else lean_rows<T, V, INIT, SEG, UPONLY, NW>(a, static_cast<int64_t>(blockIdx.x) - heavy_blocks);
}

// All-heavy levels under narrow_variant 11 / 12: the lean heavy walk alone.
template <typename T, int V, int INIT, bool UPONLY>
__global__ void __launch_bounds__(kWarpRowThreads) level_lean_warp_kernel(LevelArgs a) {
    pdl_trigger();
    lean_heavy_rows<T, V, INIT, UPONLY>(a, blockIdx.x);
}

// Narrow rows of padded lists, persistent (narrow_variant 9 and 10).  The narrow CTAs of a
// launch are capped at what the GPU holds at once, and each warp walks row groups W warps
// apart (W = warps of the narrow part).  While a group's source rows load, the warp already
// holds the next group's list extent and requests its first 4 codes, so a group
// costs only its rounds of row fetches (the row pointer -> codes chain of the next group is
// hidden behind them) and a level has no partial last wave.  The per-row arithmetic is that
// of vec_rows, so results are bit-identical to variants 6 and 7.
template <typename T, int V, int INIT>
__device__ __forceinline__ void persist_rows(const LevelArgs& a, int32_t block, int32_t nblocks) {
    // 32-bit positions and row ids: the host picks this path only for levels under 2^30 rows,
    // and node ids are below 2^29.
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int32_t narrow = static_cast<int32_t>(a.num_rows - a.num_heavy);  // heavy positions form the suffix
    const int rows_log = 5 - a.log2g;  // a warp holds 32 / G consecutive positions
    const int32_t pos_stride = (nblocks * kNarrowWarps) << rows_log;
    int32_t pos = ((block * kNarrowWarps + warp) << rows_log) + (lane >> a.log2g);
    if (pos >= narrow) return;  // no warp-wide operations below
    const int glane = lane & ((1 << a.log2g) - 1);
    const uint4* codes4 = reinterpret_cast<const uint4*>(a.entries);
    const uint32_t null_code = GRG_B200_SRC_NULL << GRG_B200_SRC_SHIFT;
    const uint4 null4 = make_uint4(null_code, null_code, null_code, null_code);
    int32_t e0, e1;
    narrow_extent(a, pos, e0, e1);
    uint4 first = (e0 >> 2) < (e1 >> 2) ? __ldg(codes4 + (e0 >> 2)) : null4;  // static list: before the wait
    pdl_wait();
    T* state = static_cast<T*>(a.state);
    const int32_t step = V << a.log2g;
    const int32_t k = static_cast<int32_t>(a.k);
    for (;;) {
        // the row id is needed only by the init value and the store, after the group's rounds
        const int32_t row = static_cast<int32_t>(level_row(a, pos));
        const int32_t npos = pos + pos_stride;  // this lane group's next position (< 2^31: narrow + stride)
        const bool more = npos < narrow;
        int32_t n0 = 0, n1 = 0;
        if (more) narrow_extent(a, npos, n0, n1);
        uint4 nfirst = null4;
        bool pending = more;  // the next group's first codes are not requested yet
        for (int32_t c = glane * V; c < k; c += step) {
            Pack<T, V> acc = init_value<T, V, INIT>(a, row, c);
            Pack<T, V> seg = zero_pack<T, V>();
            const int32_t q1 = e1 >> 2;
            uint4 cur = first;
            for (int32_t q = e0 >> 2; q < q1; ++q) {
                const uint4 nxt = q + 1 < q1 ? __ldg(codes4 + q + 1) : null4;
                const uint32_t code[4] = {cur.x, cur.y, cur.z, cur.w};
                Pack<T, V> val[4];
                bool valid[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const T* src = entry_row<T>(a, code[u]);
                    valid[u] = src != nullptr;
                    val[u] = valid[u] ? ld_ro<T, V>(src + c) : zero_pack<T, V>();
                }
                if (pending) {  // after this round's fetches are issued: waits only on n0
                    nfirst = (n0 >> 2) < (n1 >> 2) ? __ldg(codes4 + (n0 >> 2)) : null4;
                    pending = false;
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    if (code[u] & GRG_B200_SEG_START) {
                        add_into(acc, seg);
                        seg = zero_pack<T, V>();
                    }
                    if (valid[u]) add_into(seg, val[u]);
                }
                cur = nxt;
            }
            add_into(acc, seg);
            st_pack(state + static_cast<int64_t>(row) * a.ld_state + c, acc);
        }
        if (!more) return;
        if (pending) nfirst = (n0 >> 2) < (n1 >> 2) ? __ldg(codes4 + (n0 >> 2)) : null4;  // empty row
        pos = npos;
        e0 = n0;
        e1 = n1;
        first = nfirst;
    }
}

// heavy_variant 2 with narrow_variant 9 (MB = 5, 48 registers) or 10 (MB = 4, 64 registers):
// the first heavy_blocks CTAs take the heavy rows one warp each, as in level_fused_kernel; the
// other gridDim.x - heavy_blocks CTAs are the persistent narrow part.
template <typename T, int V, int INIT, int MB>
__global__ void __launch_bounds__(kNarrowThreads, MB) level_persist_kernel(LevelArgs a, int64_t heavy_blocks) {
    pdl_trigger();
    if (static_cast<int64_t>(blockIdx.x) < heavy_blocks) warp_heavy_rows<T, V, INIT>(a, blockIdx.x);
    else persist_rows<T, V, INIT>(a, static_cast<int32_t>(blockIdx.x - heavy_blocks), static_cast<int32_t>(gridDim.x - heavy_blocks));
}

// ---------------------------------------------------------------------------------------
// Fused runs of small levels (traverse_args.fuse_entries > 0)
//
// Consecutive resident levels of at most fuse_entries entries each run as one cooperative
// launch: every CTA walks the level's virtual CTAs (heavy-row CTAs first, then narrow-row
// CTAs, numbered as in level_fused_kernel), then all CTAs meet at a grid barrier before the
// next level.  Rows written earlier in the launch are read through L2 (ld.cg), so no SM can
// use a stale L1 line.  The per-row arithmetic is that of level_fused_kernel, so results are
// bit-identical to one launch per level.  The barrier wait is bounded: after
// kBarrierSpinLimit polls a CTA records kErrWaitTimeout in sync[2] and raises the abort flag
// sync[1], and every CTA leaves at its next barrier.  A cooperative launch keeps every CTA
// resident, so a correct launch never reaches the limit.
// ---------------------------------------------------------------------------------------
constexpr int kRunMaxLevels = 48;
constexpr int kBarrierSpinLimit = 1 << 22;  // polls of one barrier, each after a ~64 ns sleep

struct RunArgs {
    int32_t* sync;  // [0] barrier arrivals, [1] abort flag (both zeroed before the launch), [2] status
    int32_t num_levels;
    int64_t heavy_blocks[kRunMaxLevels];
    int64_t blocks[kRunMaxLevels];  // heavy + narrow virtual CTAs of each level
    LevelArgs lv[kRunMaxLevels];
};
static_assert(sizeof(RunArgs) <= 32000, "launch parameters above the 32 KB limit");

// Grid barrier number `phase` (1, 2, ...): false when the run is aborted (uniform per CTA).
__device__ __forceinline__ bool run_barrier(const RunArgs& p, int phase) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int good = 1;
        __threadfence();  // this CTA's rows of the level are visible before it arrives
        atomicAdd(p.sync, 1);
        const int target = phase * static_cast<int>(gridDim.x);
        volatile const int32_t* arrived = p.sync;
        volatile const int32_t* aborted = p.sync + 1;
        for (int spin = 0; *arrived < target; ++spin) {
            if (*aborted) {
                good = 0;
                break;
            }
            if (spin >= kBarrierSpinLimit) {
                atomicCAS(p.sync + 2, 0, static_cast<int32_t>(kErrWaitTimeout));
                atomicExch(p.sync + 1, 1);
                good = 0;
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

template <typename T, int V, int INIT, int MB>
__global__ void __launch_bounds__(kNarrowThreads, MB) level_run_kernel(const __grid_constant__ RunArgs p) {
    for (int i = 0; i < p.num_levels; ++i) {
        const LevelArgs& a = p.lv[i];
        const int64_t hb = p.heavy_blocks[i];
        for (int64_t vb = blockIdx.x; vb < p.blocks[i]; vb += gridDim.x) {  // the same trip count in every thread
            if (vb < hb) warp_heavy_rows<T, V, INIT, kWarpRowThreads / 32, true>(a, vb);
            else vec_rows<T, V, INIT, 1, true>(a, vb - hb);
        }
        if (i + 1 < p.num_levels && !run_barrier(p, i + 1)) return;
    }
}

// ---------------------------------------------------------------------------------------
// Mixed storage (dtype GRG_B200_MIXED)
//
// A value v is stored in 6 bytes as hi = v rounded to nearest FP32 plus a 16-bit signed
// correction lo, so that v ~= hi + lo * 2^(e(hi) - 38), where e(hi) is hi's unbiased exponent
// (FP32 subnormals use the smallest normal exponent).  |v - hi| is at most half an FP32 ulp,
// 2^(e - 24), so |lo| <= 2^14 always fits; the stored value is within 2^-39 of v relative to
// |hi| and integers below 2^39 are exact.  Decoding is exact in FP64 (24 + 15 bits fit in 53),
// every sum is accumulated in FP64 registers and rounded back to 6 bytes once per node.  A buffer of R rows and ld
// columns (ld % 4 == 0) is two planes: float hi[R * ld] followed by int16 lo[R * ld].
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t mx_exp_field(float hi) {
    const uint32_t e = (__float_as_uint(hi) >> 23) & 0xffu;
    return e == 0u ? 1u : e;
}

// 2^(e - 38) for the biased exponent field E = e + 127: 2^(E - 165) as a double.
__device__ __forceinline__ double mx_unit(float hi) {
    return __longlong_as_double(static_cast<long long>(mx_exp_field(hi) + (1023u - 165u)) << 52);
}

__device__ __forceinline__ double mx_inv_unit(float hi) {
    return __longlong_as_double(static_cast<long long>((1023u + 165u) - mx_exp_field(hi)) << 52);
}

__device__ __forceinline__ double mx_decode(float hi, short lo) {
    return static_cast<double>(hi) + static_cast<double>(lo) * mx_unit(hi);
}

__device__ __forceinline__ void mx_encode(double v, float& hi, short& lo) {
    hi = __double2float_rn(v);
    if (!isfinite(hi)) {
        lo = 0;
        return;
    }
    const double r = v - static_cast<double>(hi);  // exact
    lo = static_cast<short>(__double2int_rn(r * mx_inv_unit(hi)));  // |lo| <= 2^14
}

struct Quad {
    double v[4];
};

__device__ __forceinline__ Quad zero_quad() { return Quad{{0.0, 0.0, 0.0, 0.0}}; }

__device__ __forceinline__ void add_quad(Quad& a, const Quad& b) {
#pragma unroll
    for (int i = 0; i < 4; ++i) a.v[i] = a.v[i] + b.v[i];
}

// Four encoded columns [c, c + 4) as loaded (16-byte hi load + 8-byte lo load).
struct RawQuad {
    float4 h;
    short4 l;
};

__device__ __forceinline__ RawQuad mx_load_raw(const float* hi_row, const short* lo_row) {
    return RawQuad{__ldg(reinterpret_cast<const float4*>(hi_row)), __ldg(reinterpret_cast<const short4*>(lo_row))};
}

__device__ __forceinline__ void add_raw(Quad& a, const RawQuad& r) {
    a.v[0] = a.v[0] + mx_decode(r.h.x, r.l.x);
    a.v[1] = a.v[1] + mx_decode(r.h.y, r.l.y);
    a.v[2] = a.v[2] + mx_decode(r.h.z, r.l.z);
    a.v[3] = a.v[3] + mx_decode(r.h.w, r.l.w);
}

__device__ __forceinline__ Quad mx_load(const float* hi_row, const short* lo_row) {
    Quad q = zero_quad();
    add_raw(q, mx_load_raw(hi_row, lo_row));
    return q;
}

__device__ __forceinline__ void mx_store(float* hi_row, short* lo_row, const Quad& q) {
    float4 h;
    short4 l;
    mx_encode(q.v[0], h.x, l.x);
    mx_encode(q.v[1], h.y, l.y);
    mx_encode(q.v[2], h.z, l.z);
    mx_encode(q.v[3], h.w, l.w);
    *reinterpret_cast<float4*>(hi_row) = h;
    *reinterpret_cast<short4*>(lo_row) = l;
}

// Columns [c, c + 4) of an FP64 row with columns >= k read as zero.
__device__ __forceinline__ Quad f64_load_guarded(const double* row, int64_t c, int64_t k) {
    Quad q;
#pragma unroll
    for (int i = 0; i < 4; ++i) q.v[i] = c + i < k ? __ldg(row + c + i) : 0.0;
    return q;
}

__device__ __forceinline__ void f64_store_guarded(double* row, int64_t c, int64_t k, const Quad& q) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
        if (c + i < k) row[c + i] = q.v[i];
}

template <int INIT>
__device__ __forceinline__ Quad mx_init(const LevelArgs& a, int64_t row, int64_t c) {
    if constexpr (INIT == GRG_B200_INIT_VECTOR) {
        return f64_load_guarded(static_cast<const double*>(a.init_vector), c, a.k);
    } else if constexpr (INIT == GRG_B200_INIT_XTX) {
        const double x = __ldg(static_cast<const double*>(a.xtx_node) + row);
        return Quad{{x, x, x, x}};
    } else if constexpr (INIT == GRG_B200_INIT_MATRIX) {
        const int64_t orig = __ldg(a.node_perm + row);
        if (a.err && (orig < 0 || orig >= a.lim_state)) {
            report(a.err, kErrPerm);
            return zero_quad();
        }
        return f64_load_guarded(static_cast<const double*>(a.init_matrix) + orig * a.ld_init, c, a.k);
    } else {
        return zero_quad();
    }
}

// Encoded row named by a coded entry (hi and lo row starts); false when the entry is skipped.
__device__ __forceinline__ bool mx_entry(const LevelArgs& a, uint32_t code, const float*& hi, const short*& lo) {
    const uint32_t src = (code >> GRG_B200_SRC_SHIFT) & GRG_B200_SRC_MASK;
    const int64_t id = code & GRG_B200_ID_MASK;
    int64_t off;
    if (src == GRG_B200_SRC_STATE) {
        if (a.err && id >= a.lim_state) {
            report(a.err, kErrStateId);
            return false;
        }
        off = id * a.ld_state;
        hi = static_cast<const float*>(a.state) + off;
        lo = static_cast<const short*>(a.state_lo) + off;
        return true;
    }
    if (src == GRG_B200_SRC_INPUT) {
        if (a.err && id >= a.lim_x) {
            report(a.err, kErrInputId);
            return false;
        }
        off = id * a.ld_x;
        hi = static_cast<const float*>(a.x) + off;
        lo = static_cast<const short*>(a.x_lo) + off;
        return true;
    }
    if (src != GRG_B200_SRC_MISS || !a.use_miss) return false;
    if (a.err && id >= a.lim_miss) {
        report(a.err, kErrMissId);
        return false;
    }
    off = id * a.ld_miss;
    hi = static_cast<const float*>(a.miss) + off;
    lo = static_cast<const short*>(a.miss_lo) + off;
    return true;
}

// Generic VM-column pieces of the mixed level kernels (VM = 4: 16-byte hi + 8-byte lo loads;
// VM = 2: 8-byte hi + 4-byte lo loads, half the registers per lane, twice the lanes per row).
template <int VM>
struct MxRaw;
template <>
struct MxRaw<4> {
    float4 h;
    short4 l;
};
template <>
struct MxRaw<2> {
    float2 h;
    short2 l;
};

template <int VM>
__device__ __forceinline__ MxRaw<VM> mx_ld(const float* hi, const short* lo) {
    if constexpr (VM == 4)
        return MxRaw<4>{__ldg(reinterpret_cast<const float4*>(hi)), __ldg(reinterpret_cast<const short4*>(lo))};
    else
        return MxRaw<2>{__ldg(reinterpret_cast<const float2*>(hi)), __ldg(reinterpret_cast<const short2*>(lo))};
}

template <int VM>
__device__ __forceinline__ MxRaw<VM> mx_zero() {
    if constexpr (VM == 4) return MxRaw<4>{make_float4(0.f, 0.f, 0.f, 0.f), make_short4(0, 0, 0, 0)};
    else return MxRaw<2>{make_float2(0.f, 0.f), make_short2(0, 0)};
}

template <int VM>
__device__ __forceinline__ void mx_add(Pack<double, VM>& a, const MxRaw<VM>& r) {
    a.v[0] = a.v[0] + mx_decode(r.h.x, r.l.x);
    a.v[1] = a.v[1] + mx_decode(r.h.y, r.l.y);
    if constexpr (VM == 4) {
        a.v[2] = a.v[2] + mx_decode(r.h.z, r.l.z);
        a.v[3] = a.v[3] + mx_decode(r.h.w, r.l.w);
    }
}

template <int VM>
__device__ __forceinline__ void mx_st(float* hi, short* lo, const Pack<double, VM>& v) {
    if constexpr (VM == 4) {
        mx_store(hi, lo, Quad{{v.v[0], v.v[1], v.v[2], v.v[3]}});
    } else {
        float2 h;
        short2 l;
        mx_encode(v.v[0], h.x, l.x);
        mx_encode(v.v[1], h.y, l.y);
        *reinterpret_cast<float2*>(hi) = h;
        *reinterpret_cast<short2*>(lo) = l;
    }
}

template <int VM>
__device__ __forceinline__ Pack<double, VM> f64_ld_guarded(const double* row, int64_t c, int64_t k) {
    Pack<double, VM> q;
#pragma unroll
    for (int i = 0; i < VM; ++i) q.v[i] = c + i < k ? __ldg(row + c + i) : 0.0;
    return q;
}

template <int INIT, int VM>
__device__ __forceinline__ Pack<double, VM> mx_init_v(const LevelArgs& a, int64_t row, int64_t c) {
    if constexpr (INIT == GRG_B200_INIT_VECTOR) {
        return f64_ld_guarded<VM>(static_cast<const double*>(a.init_vector), c, a.k);
    } else if constexpr (INIT == GRG_B200_INIT_XTX) {
        return splat<double, VM>(__ldg(static_cast<const double*>(a.xtx_node) + row));
    } else if constexpr (INIT == GRG_B200_INIT_MATRIX) {
        const int64_t orig = __ldg(a.node_perm + row);
        if (a.err && (orig < 0 || orig >= a.lim_state)) {
            report(a.err, kErrPerm);
            return zero_pack<double, VM>();
        }
        return f64_ld_guarded<VM>(static_cast<const double*>(a.init_matrix) + orig * a.ld_init, c, a.k);
    } else {
        return zero_pack<double, VM>();
    }
}

// Narrow rows of padded lists in mixed storage: the ownership and code prefetch of
// level_vec_kernel with VM columns per lane; adds in list order, segment by segment.
template <int INIT, int VM>
__global__ void __launch_bounds__(kNarrowThreads, VM == 4 ? 3 : 5) level_mx_kernel(LevelArgs a) {
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int64_t narrow = a.num_rows - a.num_heavy;
    const int64_t pos = ((static_cast<int64_t>(blockIdx.x) * kNarrowWarps + warp) << (5 - a.log2g)) + (lane >> a.log2g);
    if (pos >= narrow) return;
    const int32_t e0 = __ldg(a.row_ptr + pos);
    const int32_t e1 = __ldg(a.row_ptr + pos + 1);
    const int glane = lane & ((1 << a.log2g) - 1);
    const int64_t row = level_row(a, pos);
    const uint4* codes4 = reinterpret_cast<const uint4*>(a.entries);
    const uint32_t null_code = GRG_B200_SRC_NULL << GRG_B200_SRC_SHIFT;
    const uint4 null4 = make_uint4(null_code, null_code, null_code, null_code);
    const int64_t step = static_cast<int64_t>(VM) << a.log2g;
    for (int64_t c = static_cast<int64_t>(glane) * VM; c < a.k; c += step) {
        Pack<double, VM> acc = mx_init_v<INIT, VM>(a, row, c);
        Pack<double, VM> seg = zero_pack<double, VM>();
        const int32_t q1 = e1 >> 2;
        int32_t q = e0 >> 2;
        uint4 cur = q < q1 ? __ldg(codes4 + q) : null4;
        for (; q < q1; ++q) {
            const uint4 nxt = q + 1 < q1 ? __ldg(codes4 + q + 1) : null4;
            const uint32_t code[4] = {cur.x, cur.y, cur.z, cur.w};
            MxRaw<VM> val[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const float* hi = nullptr;
                const short* lo = nullptr;
                val[u] = mx_entry(a, code[u], hi, lo) ? mx_ld<VM>(hi + c, lo + c) : mx_zero<VM>();
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (code[u] & GRG_B200_SEG_START) {
                    add_into(acc, seg);
                    seg = zero_pack<double, VM>();
                }
                mx_add<VM>(seg, val[u]);  // skipped entries decode to +0
            }
            cur = nxt;
        }
        add_into(acc, seg);
        const int64_t off = row * a.ld_state + c;
        mx_st<VM>(static_cast<float*>(a.state) + off, static_cast<short*>(a.state_lo) + off, acc);
    }
}

// Heavy rows in mixed storage, one warp each (as level_warp_kernel, padded lists).
template <int INIT, int VM>
__global__ void __launch_bounds__(kWarpRowThreads) level_mx_warp_kernel(LevelArgs a) {
    const int64_t w = static_cast<int64_t>(blockIdx.x) * (kWarpRowThreads / 32) + (threadIdx.x >> 5);
    if (w >= a.num_heavy) return;  // warp-uniform
    const int lane32 = threadIdx.x & 31;
    const int64_t pos = __ldg(a.heavy_rows + w);
    const int32_t e0 = __ldg(a.row_ptr + pos);
    const int32_t e1 = __ldg(a.row_ptr + pos + 1);
    const int64_t row = level_row(a, pos);
    const int g_lanes = 1 << a.log2g;
    const int groups = 32 >> a.log2g;
    const int glane = lane32 & (g_lanes - 1);
    const int grp = lane32 >> a.log2g;
    const uint4* codes4 = reinterpret_cast<const uint4*>(a.entries);
    const int64_t step = static_cast<int64_t>(VM) << a.log2g;
    for (int64_t base = 0; base < a.k; base += step) {  // uniform trip count across the warp
        const int64_t c = base + static_cast<int64_t>(glane) * VM;
        const bool active = c < a.k;
        Pack<double, VM> part = zero_pack<double, VM>();
        if (active) {
            for (int32_t q = (e0 >> 2) + grp; q < (e1 >> 2); q += groups) {
                const uint4 cq = __ldg(codes4 + q);
                const uint32_t code[4] = {cq.x, cq.y, cq.z, cq.w};
                MxRaw<VM> val[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const float* hi = nullptr;
                    const short* lo = nullptr;
                    val[u] = mx_entry(a, code[u], hi, lo) ? mx_ld<VM>(hi + c, lo + c) : mx_zero<VM>();
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) mx_add<VM>(part, val[u]);
            }
        }
        for (int off = 16; off >= g_lanes; off >>= 1) {
            const Pack<double, VM> other = shfl_xor_pack(part, off);
            add_into(part, other);
        }
        if (grp == 0 && active) {
            Pack<double, VM> acc = mx_init_v<INIT, VM>(a, row, c);
            add_into(acc, part);
            const int64_t o = row * a.ld_state + c;
            mx_st<VM>(static_cast<float*>(a.state) + o, static_cast<short*>(a.state_lo) + o, acc);
        }
    }
}

// Encoded copy of an FP64 matrix: dst[r, c] = src[r, c] for c < k, 0 for k <= c < ld.
__global__ void __launch_bounds__(256) mx_encode_rows_kernel(const double* src, int64_t ld_src, int64_t rows, int64_t k,
                                                             float* dst_hi, short* dst_lo, int64_t ld, int32_t log2g) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t r = t >> log2g;
    if (r >= rows) return;
    const int lane = static_cast<int>(t & ((1 << log2g) - 1));
    for (int64_t c = static_cast<int64_t>(lane) * 4; c < ld; c += static_cast<int64_t>(4) << log2g)
        mx_store(dst_hi + r * ld + c, dst_lo + r * ld + c, f64_load_guarded(src + r * ld_src, c, k));
}

// Up seeding of level 0 in mixed storage: state[r] = init(r) (+ input row for samples).
template <int INIT>
__global__ void __launch_bounds__(256) seed_up_mx_kernel(LevelArgs a, int64_t num_samples, const int32_t* s2i, int32_t by_ind) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t row = t >> a.log2g;
    if (row >= a.num_rows) return;
    const int lane = static_cast<int>(t & ((1 << a.log2g) - 1));
    int64_t xrow = row;
    if (row < num_samples && by_ind) {
        xrow = __ldg(s2i + row);
        if (a.err && (xrow < 0 || xrow >= a.lim_x)) {
            report(a.err, kErrInputId);
            return;
        }
    }
    const double* x = static_cast<const double*>(a.x);
    for (int64_t c = static_cast<int64_t>(lane) * 4; c < a.k; c += static_cast<int64_t>(4) << a.log2g) {
        Quad v = mx_init<INIT>(a, row, c);
        if (row < num_samples) add_quad(v, f64_load_guarded(x + xrow * a.ld_x, c, a.k));
        const int64_t o = row * a.ld_state + c;
        mx_store(static_cast<float*>(a.state) + o, static_cast<short*>(a.state_lo) + o, v);
    }
}

constexpr int kWideThreads = 128;
constexpr int kWideChunk = 512;  // gather-list entries staged per round

// Heavy rows, one CTA each.  Default: the CTA stages the list in chunks, entry groups of G
// lanes fetch rows independently, and the partial sums are tree-reduced in a fixed order
// (deterministic; exact whenever the data are integers).  EXACT: chunks are fetched in
// parallel but added by one lane group in list order (bit-identical to the reference).
template <typename T, int V, int INIT, bool EXACT>
__global__ void __launch_bounds__(kWideThreads) level_wide_kernel(LevelArgs a) {
    __shared__ Pack<T, V> red[kWideThreads];
    __shared__ uint32_t codes[kWideChunk];
    const int64_t pos = __ldg(a.heavy_rows + blockIdx.x);
    const int32_t e0 = __ldg(a.row_ptr + pos);
    const int32_t e1 = __ldg(a.row_ptr + pos + 1);
    const int64_t row = level_row(a, pos);
    const int g_lanes = 1 << a.log2g;
    const int groups = kWideThreads >> a.log2g;
    const int lane = threadIdx.x & (g_lanes - 1);
    const int grp = threadIdx.x >> a.log2g;
    T* state = static_cast<T*>(a.state);
    const int64_t step = static_cast<int64_t>(V) << a.log2g;
    for (int64_t base = 0; base < a.k; base += step) {  // uniform trip count across the CTA
        const int64_t c = base + static_cast<int64_t>(lane) * V;
        const bool active = c < a.k;
        if constexpr (!EXACT) {
            constexpr int UW = 4;
            Pack<T, V> part = zero_pack<T, V>();
            for (int32_t s0 = e0; s0 < e1; s0 += kWideChunk) {
                const int n = min(kWideChunk, e1 - s0);
                __syncthreads();
                for (int j = threadIdx.x; j < n; j += kWideThreads) codes[j] = __ldg(a.entries + s0 + j);
                __syncthreads();
                if (active) {
                    for (int j = grp; j < n; j += groups * UW) {
                        Pack<T, V> val[UW];
#pragma unroll
                        for (int u = 0; u < UW; ++u) {
                            const int jj = j + u * groups;
                            const T* src = jj < n ? entry_row<T>(a, codes[jj]) : nullptr;
                            val[u] = src ? ld_ro<T, V>(src + c) : zero_pack<T, V>();
                        }
#pragma unroll
                        for (int u = 0; u < UW; ++u) add_into(part, val[u]);
                    }
                }
            }
            red[threadIdx.x] = part;
            __syncthreads();
            for (int s = groups >> 1; s > 0; s >>= 1) {
                if (grp < s) {
                    Pack<T, V> other = red[threadIdx.x + (s << a.log2g)];
                    add_into(red[threadIdx.x], other);
                }
                __syncthreads();
            }
            if (grp == 0 && active) {
                Pack<T, V> acc = init_value<T, V, INIT>(a, row, c);
                add_into(acc, red[threadIdx.x]);
                st_pack(state + row * a.ld_state + c, acc);
            }
            __syncthreads();
        } else {
            Pack<T, V> acc = zero_pack<T, V>();
            Pack<T, V> seg = zero_pack<T, V>();
            if (grp == 0 && active) acc = init_value<T, V, INIT>(a, row, c);
            for (int32_t s0 = e0; s0 < e1; s0 += groups) {
                const int32_t e = s0 + grp;
                Pack<T, V> val = zero_pack<T, V>();
                uint32_t code = 0;
                if (e < e1) {
                    code = __ldg(a.entries + e);
                    const T* src = entry_row<T>(a, code);
                    if (src && active) val = ld_ro<T, V>(src + c);
                }
                red[threadIdx.x] = val;
                if (lane == 0) codes[grp] = code;
                __syncthreads();
                if (grp == 0 && active) {
                    const int n = min(groups, e1 - s0);
                    for (int i = 0; i < n; ++i) {
                        if (codes[i] & GRG_B200_SEG_START) {
                            add_into(acc, seg);
                            seg = zero_pack<T, V>();
                        }
                        add_into(seg, red[(i << a.log2g) + lane]);
                    }
                }
                __syncthreads();
            }
            if (grp == 0 && active) {
                add_into(acc, seg);
                st_pack(state + row * a.ld_state + c, acc);
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// Dataflow traversal (schedule GRG_B200_SCHEDULE_DATAFLOW): one persistent launch walks every
// level.  Warps take tasks (a heavy row, or the narrow rows of one warp) from a global
// counter in execution order, so every source of a task belongs to an earlier task that a
// running warp already holds; a row therefore waits only for its own sources, not for the
// whole previous level.  Readiness travels with the data: before the launch the rows this
// traversal writes are filled with a NaN sentinel, and a reader re-loads (from L2) any value
// that still holds it.  Every wait is bounded: after kSpinLimit retries the warp records
// kErrWaitTimeout, raises the abort flag (which every warp polls) and stops.
// ---------------------------------------------------------------------------------------
constexpr int kDfMaxLevels = 128;
constexpr int kDfThreads = 256;
constexpr int kDfGrab = 2;          // tasks taken per counter increment
constexpr int kSpinLimit = 1 << 20;  // retries of one load (each after a ~100 ns sleep)

struct DfLevel {
    const int32_t* row_ptr;
    const uint4* codes;
    const int32_t* row_ids;
    int64_t row_begin;
    int32_t num_rows;
    int32_t num_heavy;
};

struct DfArgs {
    LevelArgs a;          // shared fields: state, inputs, init, k, log2g, limits, error word
    int32_t* sync;        // [0] task counter, [1] abort flag, [2] status (zeroed before the launch)
    int32_t total_tasks;
    int32_t num_levels;
    int32_t task_begin[kDfMaxLevels + 1];
    DfLevel lv[kDfMaxLevels];
};

template <typename T>
struct SentinelBits;
template <>
struct SentinelBits<double> {
    static constexpr unsigned long long value = 0xFFF80DEADBEEF001ull;  // a quiet NaN no sum produces from finite data
};
template <>
struct SentinelBits<float> {
    static constexpr unsigned value = 0xFFC0DEADu;
};

__device__ __forceinline__ bool is_sentinel(double x) {
    return static_cast<unsigned long long>(__double_as_longlong(x)) == SentinelBits<double>::value;
}
__device__ __forceinline__ bool is_sentinel(float x) { return __float_as_uint(x) == SentinelBits<float>::value; }

template <typename T, int V>
__device__ __forceinline__ bool any_sentinel(const Pack<T, V>& p) {
    bool s = false;
#pragma unroll
    for (int i = 0; i < V; ++i) s |= is_sentinel(p.v[i]);
    return s;
}

__device__ __forceinline__ bool df_aborted(const DfArgs& p) {
    return *reinterpret_cast<volatile const int32_t*>(p.sync + 1) != 0;
}

// Re-load a state row until it no longer holds the sentinel (bounded).
template <typename T, int V>
__device__ __noinline__ Pack<T, V> df_wait(const DfArgs& p, const T* src, Pack<T, V> v) {
    for (int spin = 0; any_sentinel(v); ++spin) {
        if (spin >= kSpinLimit || df_aborted(p)) {
            if (spin >= kSpinLimit) {
                report(p.a.err, kErrWaitTimeout);
                atomicCAS(p.sync + 2, 0, kErrWaitTimeout);
            }
            atomicExch(p.sync + 1, 1);
            return zero_pack<T, V>();
        }
        __nanosleep(100);
        v = ld_l2<T, V>(src);
    }
    return v;
}

// Fetch one entry's row: state rows through L2 with the readiness check, inputs as usual.
template <typename T, int V>
__device__ __forceinline__ Pack<T, V> df_fetch(const DfArgs& p, uint32_t code, int64_t c) {
    const uint32_t src = (code >> GRG_B200_SRC_SHIFT) & GRG_B200_SRC_MASK;
    if (src == GRG_B200_SRC_STATE) {
        const T* row = entry_row<T>(p.a, code);
        if (!row) return zero_pack<T, V>();
        Pack<T, V> v = ld_l2<T, V>(row + c);
        if (any_sentinel(v)) v = df_wait<T, V>(p, row + c, v);
        return v;
    }
    const T* row = entry_row<T>(p.a, code);
    return row ? ld_ro<T, V>(row + c) : zero_pack<T, V>();
}

template <typename T, int V, int INIT>
__device__ __forceinline__ void df_narrow(const DfArgs& p, const DfLevel& L, int64_t task) {
    const LevelArgs& a = p.a;
    const int lane = threadIdx.x & 31;
    const int64_t narrow = L.num_rows - L.num_heavy;
    const int64_t pos = (task << (5 - a.log2g)) + (lane >> a.log2g);
    if (pos >= narrow) return;
    const int32_t e0 = __ldg(L.row_ptr + pos);
    const int32_t e1 = __ldg(L.row_ptr + pos + 1);
    const int glane = lane & ((1 << a.log2g) - 1);
    const int64_t row = L.row_begin + (L.row_ids ? static_cast<int64_t>(__ldg(L.row_ids + pos)) : pos);
    const uint32_t null_code = GRG_B200_SRC_NULL << GRG_B200_SRC_SHIFT;
    const uint4 null4 = make_uint4(null_code, null_code, null_code, null_code);
    T* state = static_cast<T*>(a.state);
    const int64_t step = static_cast<int64_t>(V) << a.log2g;
    for (int64_t c = static_cast<int64_t>(glane) * V; c < a.k; c += step) {
        Pack<T, V> acc = init_value<T, V, INIT>(a, row, c);
        Pack<T, V> seg = zero_pack<T, V>();
        const int32_t q1 = e1 >> 2;
        int32_t q = e0 >> 2;
        uint4 cur = q < q1 ? __ldg(L.codes + q) : null4;
        for (; q < q1; ++q) {
            const uint4 nxt = q + 1 < q1 ? __ldg(L.codes + q + 1) : null4;
            const uint32_t code[4] = {cur.x, cur.y, cur.z, cur.w};
            Pack<T, V> val[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) val[u] = df_fetch<T, V>(p, code[u], c);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (code[u] & GRG_B200_SEG_START) {
                    add_into(acc, seg);
                    seg = zero_pack<T, V>();
                }
                add_into(seg, val[u]);  // skipped entries fetch +0
            }
            cur = nxt;
        }
        add_into(acc, seg);
        st_pack(state + row * a.ld_state + c, acc);
    }
}

template <typename T, int V, int INIT>
__device__ __forceinline__ void df_heavy(const DfArgs& p, const DfLevel& L, int64_t h) {
    const LevelArgs& a = p.a;
    const int lane32 = threadIdx.x & 31;
    const int64_t pos = L.num_rows - L.num_heavy + h;
    const int32_t e0 = __ldg(L.row_ptr + pos);
    const int32_t e1 = __ldg(L.row_ptr + pos + 1);
    const int64_t row = L.row_begin + (L.row_ids ? static_cast<int64_t>(__ldg(L.row_ids + pos)) : pos);
    const int g_lanes = 1 << a.log2g;
    const int groups = 32 >> a.log2g;
    const int glane = lane32 & (g_lanes - 1);
    const int grp = lane32 >> a.log2g;
    T* state = static_cast<T*>(a.state);
    const int64_t step = static_cast<int64_t>(V) << a.log2g;
    for (int64_t base = 0; base < a.k; base += step) {  // uniform trip count across the warp
        const int64_t c = base + static_cast<int64_t>(glane) * V;
        const bool active = c < a.k;
        Pack<T, V> part = zero_pack<T, V>();
        if (active) {
            for (int32_t q = (e0 >> 2) + grp; q < (e1 >> 2); q += groups) {
                const uint4 cq = __ldg(L.codes + q);
                const uint32_t code[4] = {cq.x, cq.y, cq.z, cq.w};
                Pack<T, V> val[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) val[u] = df_fetch<T, V>(p, code[u], c);
#pragma unroll
                for (int u = 0; u < 4; ++u) add_into(part, val[u]);
            }
        }
        for (int off = 16; off >= g_lanes; off >>= 1) {
            const Pack<T, V> other = shfl_xor_pack(part, off);
            add_into(part, other);
        }
        if (grp == 0 && active) {
            Pack<T, V> acc = init_value<T, V, INIT>(a, row, c);
            add_into(acc, part);
            st_pack(state + row * a.ld_state + c, acc);
        }
    }
}

template <typename T, int V, int INIT>
__global__ void __launch_bounds__(kDfThreads, 4) dataflow_kernel(const __grid_constant__ DfArgs p) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        int32_t t0 = 0;
        if (lane == 0) t0 = df_aborted(p) ? p.total_tasks : atomicAdd(p.sync, kDfGrab);
        t0 = __shfl_sync(kFullMask, t0, 0);
        if (t0 >= p.total_tasks) return;
        const int32_t t1 = min(t0 + kDfGrab, p.total_tasks);
        for (int32_t t = t0; t < t1; ++t) {
            int lo = 0, hi = p.num_levels;  // last level whose first task is <= t
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (p.task_begin[mid] <= t) lo = mid;
                else hi = mid;
            }
            const DfLevel& L = p.lv[lo];
            const int64_t local = t - p.task_begin[lo];
            if (local < L.num_heavy) df_heavy<T, V, INIT>(p, L, local);
            else df_narrow<T, V, INIT>(p, L, local - L.num_heavy);
        }
    }
}

// Fill rows [r0, r1) of the state (ld_state columns) with the sentinel.
template <typename T>
__global__ void __launch_bounds__(256) sentinel_fill_kernel(T* state, int64_t n) {
    using Bits = typename std::conditional<std::is_same<T, double>::value, unsigned long long, unsigned>::type;
    const Bits bits = static_cast<Bits>(SentinelBits<T>::value);
    Bits* out = reinterpret_cast<Bits*>(state);
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[i] = bits;
}

// Up seeding of level 0: state[r] = init(r) (+ input row for samples).
template <typename T, int V, int INIT>
__global__ void __launch_bounds__(256) seed_up_kernel(LevelArgs a, int64_t num_samples, const int32_t* s2i, int32_t by_ind) {
    pdl_trigger();
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t row = t >> a.log2g;
    if (row >= a.num_rows) return;
    const int lane = static_cast<int>(t & ((1 << a.log2g) - 1));
    T* state = static_cast<T*>(a.state);
    int64_t xrow = row;
    if (row < num_samples && by_ind) {
        xrow = __ldg(s2i + row);
        if (a.err && (xrow < 0 || xrow >= a.lim_x)) {
            report(a.err, kErrInputId);
            return;
        }
    }
    pdl_wait();  // inputs, init values and the state it overwrites belong to earlier kernels
    const int64_t step = static_cast<int64_t>(V) << a.log2g;
    for (int64_t c = static_cast<int64_t>(lane) * V; c < a.k; c += step) {
        Pack<T, V> v = init_value<T, V, INIT>(a, row, c);
        if (row < num_samples) add_into(v, ld_ro<T, V>(static_cast<const T*>(a.x) + xrow * a.ld_x + c));
        st_pack(state + row * a.ld_state + c, v);
    }
}

struct OutArgs {
    int64_t rows;
    const int32_t* ptr;    // selector / individual CSR
    const int32_t* idx;
    const void* state;
    int64_t ld_state;
    void* out;
    int64_t ld_out;
    const void* bias;      // per output row (up) or per sample (down)
    const void* init_vector;
    int32_t bias_mode;
    int64_t k;
    int32_t log2g;
    int32_t* err;
    int64_t lim;
    const void* state_lo;  // mixed storage only
};

template <typename T, int V>
__device__ __forceinline__ void apply_bias(const OutArgs& a, int64_t r, int64_t c, Pack<T, V>& v) {
    if (a.bias_mode == GRG_B200_BIAS_XTX) {
        const T b = __ldg(static_cast<const T*>(a.bias) + r);
#pragma unroll
        for (int i = 0; i < V; ++i) v.v[i] = add_rn(v.v[i], b);
    } else if (a.bias_mode == GRG_B200_BIAS_VECTOR) {
        const T b = __ldg(static_cast<const T*>(a.bias) + r);
        const Pack<T, V> iv = ld_ro<T, V>(static_cast<const T*>(a.init_vector) + c);
#pragma unroll
        for (int i = 0; i < V; ++i) v.v[i] = add_rn(v.v[i], mul_rn(b, iv.v[i]));
    }
}

// out[r] = sum over idx[ptr[r]..ptr[r+1]) of state rows (from zero, in order) + bias.
template <typename T, int V, bool BIAS_PER_ENTRY>
__global__ void __launch_bounds__(256) gather_out_kernel(OutArgs a) {
    pdl_wait();
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t r = t >> a.log2g;
    if (r >= a.rows) return;
    const int lane = static_cast<int>(t & ((1 << a.log2g) - 1));
    const int32_t e0 = __ldg(a.ptr + r), e1 = __ldg(a.ptr + r + 1);
    const T* state = static_cast<const T*>(a.state);
    T* out = static_cast<T*>(a.out);
    const int64_t step = static_cast<int64_t>(V) << a.log2g;
    for (int64_t c = static_cast<int64_t>(lane) * V; c < a.k; c += step) {
        Pack<T, V> s = zero_pack<T, V>();
        for (int32_t e = e0; e < e1; ++e) {
            const int64_t n = __ldg(a.idx + e);
            if (a.err && (n < 0 || n >= a.lim)) {
                report(a.err, kErrSelector);
                continue;
            }
            Pack<T, V> v = ld_ro<T, V>(state + n * a.ld_state + c);
            if constexpr (BIAS_PER_ENTRY) apply_bias<T, V>(a, n, c, v);  // down by individual
            add_into(s, v);
        }
        if constexpr (!BIAS_PER_ENTRY) apply_bias<T, V>(a, r, c, s);
        st_pack(out + r * a.ld_out + c, s);
    }
}

// Down output without grouping: out[s] = state[s] + bias[s].
template <typename T, int V>
__global__ void __launch_bounds__(256) copy_out_kernel(OutArgs a) {
    pdl_wait();
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t r = t >> a.log2g;
    if (r >= a.rows) return;
    const int lane = static_cast<int>(t & ((1 << a.log2g) - 1));
    const T* state = static_cast<const T*>(a.state);
    T* out = static_cast<T*>(a.out);
    const int64_t step = static_cast<int64_t>(V) << a.log2g;
    for (int64_t c = static_cast<int64_t>(lane) * V; c < a.k; c += step) {
        Pack<T, V> v = ld_ro<T, V>(state + r * a.ld_state + c);
        apply_bias<T, V>(a, r, c, v);
        st_pack(out + r * a.ld_out + c, v);
    }
}

// All nodes in original order: out[j] = state[inv_perm[j]].
template <typename T, int V>
__global__ void __launch_bounds__(256) emit_all_kernel(OutArgs a) {
    pdl_wait();
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t j = t >> a.log2g;
    if (j >= a.rows) return;
    const int lane = static_cast<int>(t & ((1 << a.log2g) - 1));
    const int64_t n = __ldg(a.idx + j);
    if (a.err && (n < 0 || n >= a.lim)) {
        report(a.err, kErrPerm);
        return;
    }
    const T* state = static_cast<const T*>(a.state);
    T* out = static_cast<T*>(a.out);
    const int64_t step = static_cast<int64_t>(V) << a.log2g;
    for (int64_t c = static_cast<int64_t>(lane) * V; c < a.k; c += step)
        st_pack(out + j * a.ld_out + c, ld_ro<T, V>(state + n * a.ld_state + c));
}

// Output kernels for mixed storage: decode to FP64, 4 columns per lane, columns >= k skipped.
__device__ __forceinline__ void mx_apply_bias(const OutArgs& a, int64_t r, int64_t c, Quad& v) {
    if (a.bias_mode == GRG_B200_BIAS_XTX) {
        const double b = __ldg(static_cast<const double*>(a.bias) + r);
#pragma unroll
        for (int i = 0; i < 4; ++i) v.v[i] = __dadd_rn(v.v[i], b);
    } else if (a.bias_mode == GRG_B200_BIAS_VECTOR) {
        const double b = __ldg(static_cast<const double*>(a.bias) + r);
        const Quad iv = f64_load_guarded(static_cast<const double*>(a.init_vector), c, a.k);
#pragma unroll
        for (int i = 0; i < 4; ++i) v.v[i] = __dadd_rn(v.v[i], __dmul_rn(b, iv.v[i]));
    }
}

__device__ __forceinline__ Quad mx_state_row(const OutArgs& a, int64_t n, int64_t c) {
    const int64_t o = n * a.ld_state + c;
    return mx_load(static_cast<const float*>(a.state) + o, static_cast<const short*>(a.state_lo) + o);
}

template <bool BIAS_PER_ENTRY>
__global__ void __launch_bounds__(256) gather_out_mx_kernel(OutArgs a) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t r = t >> a.log2g;
    if (r >= a.rows) return;
    const int lane = static_cast<int>(t & ((1 << a.log2g) - 1));
    const int32_t e0 = __ldg(a.ptr + r), e1 = __ldg(a.ptr + r + 1);
    double* out = static_cast<double*>(a.out);
    for (int64_t c = static_cast<int64_t>(lane) * 4; c < a.k; c += static_cast<int64_t>(4) << a.log2g) {
        Quad s = zero_quad();
        for (int32_t e = e0; e < e1; ++e) {
            const int64_t n = __ldg(a.idx + e);
            if (a.err && (n < 0 || n >= a.lim)) {
                report(a.err, kErrSelector);
                continue;
            }
            Quad v = mx_state_row(a, n, c);
            if constexpr (BIAS_PER_ENTRY) mx_apply_bias(a, n, c, v);
            add_quad(s, v);
        }
        if constexpr (!BIAS_PER_ENTRY) mx_apply_bias(a, r, c, s);
        f64_store_guarded(out + r * a.ld_out, c, a.k, s);
    }
}

__global__ void __launch_bounds__(256) copy_out_mx_kernel(OutArgs a) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t r = t >> a.log2g;
    if (r >= a.rows) return;
    const int lane = static_cast<int>(t & ((1 << a.log2g) - 1));
    double* out = static_cast<double*>(a.out);
    for (int64_t c = static_cast<int64_t>(lane) * 4; c < a.k; c += static_cast<int64_t>(4) << a.log2g) {
        Quad v = mx_state_row(a, r, c);
        mx_apply_bias(a, r, c, v);
        f64_store_guarded(out + r * a.ld_out, c, a.k, v);
    }
}

__global__ void __launch_bounds__(256) emit_all_mx_kernel(OutArgs a) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t j = t >> a.log2g;
    if (j >= a.rows) return;
    const int lane = static_cast<int>(t & ((1 << a.log2g) - 1));
    const int64_t n = __ldg(a.idx + j);
    if (a.err && (n < 0 || n >= a.lim)) {
        report(a.err, kErrPerm);
        return;
    }
    double* out = static_cast<double*>(a.out);
    for (int64_t c = static_cast<int64_t>(lane) * 4; c < a.k; c += static_cast<int64_t>(4) << a.log2g)
        f64_store_guarded(out + j * a.ld_out, c, a.k, mx_state_row(a, n, c));
}

// ---------------------------------------------------------------------------------------
// Host-side launch helpers
// ---------------------------------------------------------------------------------------
struct Shape {
    int vec;    // V
    int log2g;  // lanes per row = 1 << log2g
};

bool aligned(const void* p, int bytes) { return p == nullptr || (reinterpret_cast<uintptr_t>(p) % bytes) == 0; }

Shape choose_shape(const grg_b200_traverse_args* a) {
    if (a->dtype == GRG_B200_MIXED) {  // 4 columns per lane (16-byte hi + 8-byte lo loads)
        const int64_t cols = (a->k + 3) / 4;
        int log2g = 0;
        while ((1 << log2g) < cols && log2g < 5) ++log2g;
        return {4, log2g};
    }
    const int esize = a->dtype == GRG_B200_F64 ? 8 : 4;
    const int64_t lds[] = {a->ld_state, a->ld_input, a->ld_output, a->use_miss ? a->ld_miss : 0, a->ld_init};
    const void* ptrs[] = {a->state, a->input, a->output, a->use_miss ? a->miss : nullptr, a->init_vector, a->init_matrix};
    int vec = 1;
    const int candidates[] = {4, 2};
    for (int v : candidates) {
        if (a->dtype == GRG_B200_F64 && v == 4) continue;
        bool ok = a->k % v == 0;
        for (int64_t ld : lds) ok = ok && (ld % v == 0);
        for (const void* p : ptrs) ok = ok && aligned(p, v * esize);
        if (ok) {
            vec = v;
            break;
        }
    }
    const int64_t cols = (a->k + vec - 1) / vec;
    int log2g = 0;
    while ((1 << log2g) < cols && log2g < 5) ++log2g;
    return {vec, log2g};
}

dim3 grid_for(int64_t rows, int log2g, int threads) {
    const int64_t total = rows << log2g;
    return dim3(static_cast<unsigned>((total + threads - 1) / threads));
}

int validate_common(const grg_b200_traverse_args* a) {
    if (!a) return fail(GRG_B200_ERR_INVALID, "args is NULL");
    if (a->dtype != GRG_B200_F64 && a->dtype != GRG_B200_F32 && a->dtype != GRG_B200_MIXED)
        return fail(GRG_B200_ERR_INVALID, "unknown dtype %d", a->dtype);
    if (a->dtype == GRG_B200_MIXED) {
        if (a->ld_state % 4 != 0 || !aligned(a->state, 16))
            return fail(GRG_B200_ERR_INVALID, "mixed state needs ld_state %% 4 == 0 and a 16-byte aligned base");
        if (a->exact_order) return fail(GRG_B200_ERR_UNSUPPORTED, "mixed storage has no exact-order mode");
        if (a->direction == GRG_B200_DOWN) {
            const int64_t need = GRG_B200_MIX_BYTES(a->num_mutations, a->ld_state) * (a->use_miss ? 2 : 1);
            if (!a->mix_scratch || !aligned(a->mix_scratch, 16) || a->mix_scratch_bytes < need)
                return fail(GRG_B200_ERR_INVALID, "mixed down needs a 16-byte aligned mix_scratch of %lld bytes (got %lld)",
                            (long long)need, (long long)a->mix_scratch_bytes);
        }
    }
    if (a->k < 1) return fail(GRG_B200_ERR_INVALID, "k must be >= 1, got %lld", (long long)a->k);
    if (a->ld_state < a->k) return fail(GRG_B200_ERR_INVALID, "ld_state %lld < k %lld", (long long)a->ld_state, (long long)a->k);
    if (!a->state) return fail(GRG_B200_ERR_INVALID, "state is NULL");
    if (a->num_nodes > (int64_t)GRG_B200_MAX_ID + 1 || a->num_mutations > (int64_t)GRG_B200_MAX_ID + 1)
        return fail(GRG_B200_ERR_UNSUPPORTED, "node/mutation counts above %u are not supported", GRG_B200_MAX_ID + 1u);
    if (a->init_mode < 0 || a->init_mode > 3) return fail(GRG_B200_ERR_INVALID, "unknown init_mode %d", a->init_mode);
    if (a->narrow_variant < 0 || a->narrow_variant >= GRG_B200_NARROW_VARIANTS)
        return fail(GRG_B200_ERR_INVALID, "narrow_variant %d outside [0, %d)", a->narrow_variant, GRG_B200_NARROW_VARIANTS);
    if (a->heavy_variant < 0 || a->heavy_variant > 3) return fail(GRG_B200_ERR_INVALID, "heavy_variant %d outside [0, 3]", a->heavy_variant);
    if (a->narrow_split < -1 || a->narrow_split > 3) return fail(GRG_B200_ERR_INVALID, "narrow_split %d outside [-1, 3]", a->narrow_split);
    if (a->persist_ctas < 0) return fail(GRG_B200_ERR_INVALID, "persist_ctas must be >= 0, got %d", a->persist_ctas);
    if (a->fuse_entries < 0) return fail(GRG_B200_ERR_INVALID, "fuse_entries must be >= 0, got %lld", (long long)a->fuse_entries);
    if (a->schedule != GRG_B200_SCHEDULE_LEVELS && a->schedule != GRG_B200_SCHEDULE_DATAFLOW)
        return fail(GRG_B200_ERR_INVALID, "unknown schedule %d", a->schedule);
    if (a->init_mode == GRG_B200_INIT_VECTOR && !a->init_vector) return fail(GRG_B200_ERR_INVALID, "init_vector is NULL");
    if (a->init_mode == GRG_B200_INIT_XTX && !a->xtx_node) return fail(GRG_B200_ERR_INVALID, "xtx_node is NULL");
    if (a->init_mode == GRG_B200_INIT_MATRIX && (!a->init_matrix || !a->node_perm || a->ld_init < a->k))
        return fail(GRG_B200_ERR_INVALID, "init_matrix/node_perm missing or ld_init < k");
    if (a->bias_mode < 0 || a->bias_mode > 2) return fail(GRG_B200_ERR_INVALID, "unknown bias_mode %d", a->bias_mode);
    if (a->bias_mode != GRG_B200_BIAS_NONE && !a->endpoint_bias) return fail(GRG_B200_ERR_INVALID, "endpoint_bias is NULL");
    if (a->bias_mode == GRG_B200_BIAS_VECTOR && !a->init_vector) return fail(GRG_B200_ERR_INVALID, "init_vector is NULL");
    return GRG_B200_OK;
}

LevelArgs level_args(const grg_b200_traverse_args* a, const Shape& sh) {
    LevelArgs la{};
    la.use_miss = a->direction == GRG_B200_DOWN && a->use_miss;
    la.state = a->state;
    la.ld_state = a->ld_state;
    la.x = a->input;
    la.ld_x = a->ld_input;
    la.miss = a->miss;
    la.ld_miss = a->ld_miss;
    la.init_vector = a->init_vector;
    la.init_matrix = a->init_matrix;
    la.ld_init = a->ld_init;
    la.node_perm = a->node_perm;
    la.xtx_node = a->xtx_node;
    la.k = a->k;
    la.log2g = sh.log2g;
    la.err = a->error_word;
    la.lim_state = a->num_nodes;
    la.lim_x = a->direction == GRG_B200_UP ? (a->by_individual ? a->num_individuals : a->num_samples) : a->num_mutations;
    la.lim_miss = a->num_mutations;
    la.up = a->direction == GRG_B200_UP;
    if (a->dtype == GRG_B200_MIXED) {
        la.state_lo = static_cast<char*>(a->state) + GRG_B200_MIX_PLANE(a->num_nodes * a->ld_state * 4);
        if (a->direction == GRG_B200_DOWN) {  // levels read the encoded copies in mix_scratch
            char* base = static_cast<char*>(a->mix_scratch);
            const int64_t hi_bytes = GRG_B200_MIX_PLANE(a->num_mutations * a->ld_state * 4);
            const int64_t one = GRG_B200_MIX_BYTES(a->num_mutations, a->ld_state);
            la.x = base;
            la.x_lo = base + hi_bytes;
            la.ld_x = a->ld_state;
            la.miss = base + one;
            la.miss_lo = base + one + hi_bytes;
            la.ld_miss = a->ld_state;
        }
    }
    return la;
}

// Streaming multiprocessors of the current device (looked up once per device).
int device_sm_count(int* out) {
    static std::atomic<int> cache[64];
    int device = 0;
    GRG_CUDA_TRY(cudaGetDevice(&device));
    if (device < 0 || device >= 64) return fail(GRG_B200_ERR_UNSUPPORTED, "device ordinal %d above 63", device);
    int sms = cache[device].load(std::memory_order_relaxed);
    if (sms <= 0) {
        GRG_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        cache[device].store(sms, std::memory_order_relaxed);
    }
    *out = sms > 0 ? sms : 1;
    return GRG_B200_OK;
}

// Persistent narrow part (narrow_variant 9 / 10, no row split): heavy_blocks CTAs for heavy
// rows, then at most what the GPU holds at once (SMs x CTAs per SM of the register budget)
// for the narrow rows.
template <typename T, int V>
int launch_persist(const LevelArgs& la, int init_mode, int variant, int64_t heavy_blocks, int64_t narrow_ctas, int persist_ctas,
                   bool pdl, cudaStream_t s) {
    int sms = 0;
    const int rc = device_sm_count(&sms);
    if (rc) return rc;
    const int64_t cap = persist_ctas > 0 ? persist_ctas : static_cast<int64_t>(sms) * (variant == 9 ? 5 : 4);
    const dim3 grid(static_cast<unsigned>(heavy_blocks + (narrow_ctas < cap ? narrow_ctas : cap)));
#define GRG_PERSIST(INIT)                                                                                                   \
    if (variant == 9) GRG_CUDA_TRY(launch_k(pdl, s, grid, kNarrowThreads, level_persist_kernel<T, V, INIT, 5>, la, heavy_blocks)); \
    else GRG_CUDA_TRY(launch_k(pdl, s, grid, kNarrowThreads, level_persist_kernel<T, V, INIT, 4>, la, heavy_blocks));
    switch (init_mode) {
        case 0: GRG_PERSIST(0) break;
        case 1: GRG_PERSIST(1) break;
        case 2: GRG_PERSIST(2) break;
        default: GRG_PERSIST(3) break;
    }
#undef GRG_PERSIST
    GRG_LAUNCH_CHECK("level_persist_kernel");
    return GRG_B200_OK;
}

template <typename T, int V>
int launch_level_typed(const LevelArgs& la, int init_mode, bool exact, int variant, int heavy_variant, int persist_ctas, bool pdl,
                       cudaStream_t s) {
    const int64_t narrow = la.num_rows - la.num_heavy;  // heavy positions form the suffix
    // the lean walks (11, 12) serve launches without an error word and without row splits;
    // others fall back to variant 7's kernels
    const bool lean = variant >= 11 && la.err == nullptr && !exact && heavy_variant == 2 &&
                      la.ld_state < (int64_t{1} << 32) && la.ld_x < (int64_t{1} << 32) && la.ld_miss < (int64_t{1} << 32);
    // variants 15 and 16 fall back to 12 in 4-warp CTAs, the others in 8-warp ones
    const int fallback_nw = variant == 15 || variant == 16 ? 4 : kNarrowWarps;
    if (variant >= 13 && variant <= 16) {  // entry-parallel narrow rows where the shape allows it, else as 12
        constexpr int C = Chunk32<T>::C;
        const bool common = lean && narrow > 0 && la.log2s == 0 && init_mode == GRG_B200_INIT_NONE;
        // 32-byte chunks: k = 2^n chunks of C columns (the shape's V = C / 2 columns per lane)
        const bool chunks = common && V == C / 2 && la.log2g >= 1 && (int64_t{V} << la.log2g) == la.k && la.ld_state % C == 0 &&
                            la.ld_x % C == 0 && (!la.use_miss || la.ld_miss % C == 0) && aligned(la.state, 32) && aligned(la.x, 32) &&
                            (!la.use_miss || aligned(la.miss, 32));
        // k below a chunk: one chunk lane of the shape's V = k columns (the shape's alignment)
        const bool narrow_k = common && !chunks && V < C && la.log2g == 0 && la.k == V;
        if (chunks || narrow_k) {
            const int nw = variant == 15 ? 4 : (variant == 16 ? 2 : kNarrowWarps);  // warps per CTA; heavy rows: one each
            const int64_t heavy_blocks = (la.num_heavy + nw - 1) / nw;
            const int lg = la.log2g + (chunks ? 0 : 1);  // log2 of a row's 2W lanes
            const int log2w = lg - 1;                    // one entry slot: W lanes per short row
            const int64_t long_rows = narrow - la.short_rows;
            const int64_t long_warps = (long_rows + (32 >> lg) - 1) >> (5 - lg);
            const int64_t short_warps = (la.short_rows + (32 >> log2w) - 1) >> (5 - log2w);
            const int64_t long_blocks = (long_warps + nw - 1) / nw;
            const dim3 grid(static_cast<unsigned>(heavy_blocks + long_blocks + (short_warps + nw - 1) / nw));
#define GRG_ENTRY(KERNEL, CW)                                                                                                   \
    if (la.up) GRG_CUDA_TRY(launch_k(pdl, s, grid, kNarrowThreads, KERNEL<T, 0, true, CW>, la, heavy_blocks, long_blocks)); \
    else GRG_CUDA_TRY(launch_k(pdl, s, grid, kNarrowThreads, KERNEL<T, 0, false, CW>, la, heavy_blocks, long_blocks));
            if (variant == 13) {
                if (chunks) { GRG_ENTRY(level_entry_kernel, C) } else { GRG_ENTRY(level_entry_kernel, V) }
            } else if (variant == 14) {
                if (chunks) { GRG_ENTRY(level_entry_pre_kernel, C) } else { GRG_ENTRY(level_entry_pre_kernel, V) }
            } else {
#define GRG_ENTRY_NW(CW, NW)                                                                                                        \
    if (la.up) GRG_CUDA_TRY(launch_k(pdl, s, grid, 32 * NW, level_entry_pre_kernel<T, 0, true, CW, NW>, la, heavy_blocks, long_blocks)); \
    else GRG_CUDA_TRY(launch_k(pdl, s, grid, 32 * NW, level_entry_pre_kernel<T, 0, false, CW, NW>, la, heavy_blocks, long_blocks));
                if (variant == 15) {
                    if (chunks) { GRG_ENTRY_NW(C, 4) } else { GRG_ENTRY_NW(V, 4) }
                } else {
                    if (chunks) { GRG_ENTRY_NW(C, 2) } else { GRG_ENTRY_NW(V, 2) }
                }
#undef GRG_ENTRY_NW
            }
#undef GRG_ENTRY
            GRG_LAUNCH_CHECK("level_entry_kernel");
            return GRG_B200_OK;
        }
        variant = 12;
    }
    if (variant == 11 || variant == 12) {
        if (lean && narrow > 0 && la.log2s == 0 && variant == 12 && fallback_nw == 4) {
            const int64_t heavy_blocks = (la.num_heavy + 3) / 4;
            const int64_t warps = (narrow + (32 >> la.log2g) - 1) >> (5 - la.log2g);
            const dim3 grid(static_cast<unsigned>(heavy_blocks + (warps + 3) / 4));
#define GRG_LEAN4(INIT)                                                                                                   \
    if (la.up) GRG_CUDA_TRY(launch_k(pdl, s, grid, 128, level_lean_kernel<T, V, INIT, false, true, 4>, la, heavy_blocks)); \
    else GRG_CUDA_TRY(launch_k(pdl, s, grid, 128, level_lean_kernel<T, V, INIT, false, false, 4>, la, heavy_blocks));
            switch (init_mode) {
                case 0: GRG_LEAN4(0) break;
                case 1: GRG_LEAN4(1) break;
                case 2: GRG_LEAN4(2) break;
                default: GRG_LEAN4(3) break;
            }
#undef GRG_LEAN4
            GRG_LAUNCH_CHECK("level_lean_kernel");
            return GRG_B200_OK;
        }
        if (lean && narrow > 0 && la.log2s == 0) {
            constexpr int rows_per_cta = kWarpRowThreads / 32;
            const int64_t heavy_blocks = (la.num_heavy + rows_per_cta - 1) / rows_per_cta;
            const int64_t warps = (narrow + (32 >> la.log2g) - 1) >> (5 - la.log2g);
            const dim3 grid(static_cast<unsigned>(heavy_blocks + (warps + kNarrowWarps - 1) / kNarrowWarps));
#define GRG_LEAN(INIT)                                                                                                                if (variant == 11) {                                                                                                                  if (la.up) GRG_CUDA_TRY(launch_k(pdl, s, grid, kNarrowThreads, level_lean_kernel<T, V, INIT, true, true>, la, heavy_blocks));          else GRG_CUDA_TRY(launch_k(pdl, s, grid, kNarrowThreads, level_lean_kernel<T, V, INIT, true, false>, la, heavy_blocks));            } else {                                                                                                                              if (la.up) GRG_CUDA_TRY(launch_k(pdl, s, grid, kNarrowThreads, level_lean_kernel<T, V, INIT, false, true>, la, heavy_blocks));         else GRG_CUDA_TRY(launch_k(pdl, s, grid, kNarrowThreads, level_lean_kernel<T, V, INIT, false, false>, la, heavy_blocks));           }
            switch (init_mode) {
                case 0: GRG_LEAN(0) break;
                case 1: GRG_LEAN(1) break;
                case 2: GRG_LEAN(2) break;
                default: GRG_LEAN(3) break;
            }
#undef GRG_LEAN
            GRG_LAUNCH_CHECK("level_lean_kernel");
            return GRG_B200_OK;
        }
        if (lean && narrow == 0 && la.num_heavy > 0) {
            constexpr int rows_per_cta = kWarpRowThreads / 32;
            const dim3 grid(static_cast<unsigned>((la.num_heavy + rows_per_cta - 1) / rows_per_cta));
#define GRG_LEAN_WARP(INIT)                                                                                                            if (la.up) GRG_CUDA_TRY(launch_k(pdl, s, grid, kWarpRowThreads, level_lean_warp_kernel<T, V, INIT, true>, la));                    else GRG_CUDA_TRY(launch_k(pdl, s, grid, kWarpRowThreads, level_lean_warp_kernel<T, V, INIT, false>, la));
            switch (init_mode) {
                case 0: GRG_LEAN_WARP(0) break;
                case 1: GRG_LEAN_WARP(1) break;
                case 2: GRG_LEAN_WARP(2) break;
                default: GRG_LEAN_WARP(3) break;
            }
#undef GRG_LEAN_WARP
            GRG_LAUNCH_CHECK("level_lean_warp_kernel");
            return GRG_B200_OK;
        }
        variant = 7;
    }
    const bool padded_variant = variant >= 6 && variant <= 10;
    const bool persist = (variant == 9 || variant == 10) && la.log2s == 0 && la.num_rows < (int64_t{1} << 30);
    // fused launch, except for all-heavy levels (e.g. down level 0, where every sample row is
    // heavy): those run the warp kernel alone at its higher occupancy (40 registers, 6 CTAs/SM)
    if (padded_variant && heavy_variant == 2 && !exact && narrow > 0) {
        constexpr int rows_per_cta = kWarpRowThreads / 32;
        const int64_t heavy_blocks = (la.num_heavy + rows_per_cta - 1) / rows_per_cta;
        const int lg = la.log2g + la.log2s;
        const int64_t warps = (narrow + (32 >> lg) - 1) >> (5 - lg);
        if (persist)
            return launch_persist<T, V>(la, init_mode, variant, heavy_blocks, (warps + kNarrowWarps - 1) / kNarrowWarps, persist_ctas,
                                        pdl, s);
        const dim3 grid(static_cast<unsigned>(heavy_blocks + (warps + kNarrowWarps - 1) / kNarrowWarps));
#define GRG_FUSED_MB(INIT, MB)                                                                                 \
    if (la.log2s > 0) GRG_CUDA_TRY(launch_k(pdl, s, grid, kNarrowThreads, level_fused_kernel<T, V, INIT, true, MB>, la, heavy_blocks)); \
    else GRG_CUDA_TRY(launch_k(pdl, s, grid, kNarrowThreads, level_fused_kernel<T, V, INIT, false, MB>, la, heavy_blocks));
#define GRG_FUSED(INIT)                                                                                  \
    if (variant == 8) {                                                                                  \
        if (la.log2s > 0) GRG_CUDA_TRY(launch_k(pdl, s, grid, kNarrowThreads, level_fused_kernel<T, V, INIT, true, 6>, la, heavy_blocks)); \
        else GRG_CUDA_TRY(launch_k(pdl, s, grid, kNarrowThreads, level_fused_kernel<T, V, INIT, false, 3, 2>, la, heavy_blocks));          \
    } else if (variant == 7 || variant == 9 || variant == 10) {                                          \
        GRG_FUSED_MB(INIT, 5)                                                                            \
    } else {                                                                                             \
        GRG_FUSED_MB(INIT, 6)                                                                            \
    }
        switch (init_mode) {
            case 0: GRG_FUSED(0) break;
            case 1: GRG_FUSED(1) break;
            case 2: GRG_FUSED(2) break;
            default: GRG_FUSED(3) break;
        }
#undef GRG_FUSED
#undef GRG_FUSED_MB
        GRG_LAUNCH_CHECK("level_fused_kernel");
        return GRG_B200_OK;
    }
    if (narrow > 0 && padded_variant && la.log2s > 0) {  // split rows: the fused kernel without heavy blocks
        const int lg = la.log2g + la.log2s;
        const int64_t warps = (narrow + (32 >> lg) - 1) >> (5 - lg);
        const dim3 grid(static_cast<unsigned>((warps + kNarrowWarps - 1) / kNarrowWarps));
        switch (init_mode) {
            case 0: GRG_CUDA_TRY(launch_k(pdl, s, grid, kNarrowThreads, level_fused_kernel<T, V, 0, true, 6>, la, 0)); break;
            case 1: GRG_CUDA_TRY(launch_k(pdl, s, grid, kNarrowThreads, level_fused_kernel<T, V, 1, true, 6>, la, 0)); break;
            case 2: GRG_CUDA_TRY(launch_k(pdl, s, grid, kNarrowThreads, level_fused_kernel<T, V, 2, true, 6>, la, 0)); break;
            default: GRG_CUDA_TRY(launch_k(pdl, s, grid, kNarrowThreads, level_fused_kernel<T, V, 3, true, 6>, la, 0)); break;
        }
        GRG_LAUNCH_CHECK("level_fused_kernel(split)");
    } else if (narrow > 0 && persist) {
        const int64_t warps = (narrow + (32 >> la.log2g) - 1) >> (5 - la.log2g);
        const int rc = launch_persist<T, V>(la, init_mode, variant, 0, (warps + kNarrowWarps - 1) / kNarrowWarps, persist_ctas, pdl, s);
        if (rc) return rc;
    } else if (narrow > 0 && padded_variant) {
        const int lg = la.log2g;
        const int64_t warps = (narrow + (32 >> lg) - 1) >> (5 - lg);
        const dim3 grid(static_cast<unsigned>((warps + kNarrowWarps - 1) / kNarrowWarps));
#define GRG_VEC(INIT)                                                                      \
    if (variant == 8) GRG_CUDA_TRY(launch_k(pdl, s, grid, kNarrowThreads, level_vec_kernel<T, V, INIT, 3, 2>, la)); \
    else if (variant == 7 || variant == 9 || variant == 10) GRG_CUDA_TRY(launch_k(pdl, s, grid, kNarrowThreads, level_vec_kernel<T, V, INIT, 5>, la)); \
    else GRG_CUDA_TRY(launch_k(pdl, s, grid, kNarrowThreads, level_vec_kernel<T, V, INIT, 6>, la));
        switch (init_mode) {
            case 0: GRG_VEC(0) break;
            case 1: GRG_VEC(1) break;
            case 2: GRG_VEC(2) break;
            default: GRG_VEC(3) break;
        }
#undef GRG_VEC
        GRG_LAUNCH_CHECK("level_vec_kernel");
    } else if (narrow > 0 && variant == 4) {
        const int64_t warps = (narrow + (32 >> la.log2g) - 1) >> (5 - la.log2g);
        const dim3 grid(static_cast<unsigned>((warps + kAsyncWarps - 1) / kAsyncWarps));
        switch (init_mode) {
            case 0: level_async_kernel<T, V, 0><<<grid, kAsyncThreads, 0, s>>>(la); break;
            case 1: level_async_kernel<T, V, 1><<<grid, kAsyncThreads, 0, s>>>(la); break;
            case 2: level_async_kernel<T, V, 2><<<grid, kAsyncThreads, 0, s>>>(la); break;
            default: level_async_kernel<T, V, 3><<<grid, kAsyncThreads, 0, s>>>(la); break;
        }
        GRG_LAUNCH_CHECK("level_async_kernel");
    } else if (narrow > 0) {
        const int64_t warps = (narrow + (32 >> la.log2g) - 1) >> (5 - la.log2g);
        const dim3 grid(static_cast<unsigned>((warps + kNarrowWarps - 1) / kNarrowWarps));
#define GRG_NARROW(INIT, U, ST, MB) level_narrow_kernel<T, V, INIT, U, ST, MB><<<grid, kNarrowThreads, 0, s>>>(la)
#define GRG_NARROW_INIT(U, ST, MB)                  \
    switch (init_mode) {                            \
        case 0: GRG_NARROW(0, U, ST, MB); break;    \
        case 1: GRG_NARROW(1, U, ST, MB); break;    \
        case 2: GRG_NARROW(2, U, ST, MB); break;    \
        default: GRG_NARROW(3, U, ST, MB); break;   \
    }
        switch (variant) {
            case 1: GRG_NARROW_INIT(8, false, 1) break;
            case 2: GRG_NARROW_INIT(4, true, 1) break;
            case 3: GRG_NARROW_INIT(16, true, 1) break;
            case 5: GRG_NARROW_INIT(4, false, 8) break;
            default: GRG_NARROW_INIT(4, false, 1) break;
        }
#undef GRG_NARROW_INIT
#undef GRG_NARROW
        GRG_LAUNCH_CHECK("level_narrow_kernel");
    }
    if (la.num_heavy > 0 && !exact && heavy_variant == 3) {
        constexpr int wpc = 32;
        const dim3 grid(static_cast<unsigned>((la.num_heavy + wpc - 1) / wpc));
        switch (init_mode) {
            case 0: GRG_CUDA_TRY(launch_k(pdl, s, grid, wpc * 32, level_warp_kernel<T, V, 0, wpc>, la)); break;
            case 1: GRG_CUDA_TRY(launch_k(pdl, s, grid, wpc * 32, level_warp_kernel<T, V, 1, wpc>, la)); break;
            case 2: GRG_CUDA_TRY(launch_k(pdl, s, grid, wpc * 32, level_warp_kernel<T, V, 2, wpc>, la)); break;
            default: GRG_CUDA_TRY(launch_k(pdl, s, grid, wpc * 32, level_warp_kernel<T, V, 3, wpc>, la)); break;
        }
        GRG_LAUNCH_CHECK("level_warp_kernel(32 rows per CTA)");
    } else if (la.num_heavy > 0 && !exact && heavy_variant >= 1) {
        constexpr int rows_per_cta = kWarpRowThreads / 32;
        const dim3 grid(static_cast<unsigned>((la.num_heavy + rows_per_cta - 1) / rows_per_cta));
        switch (init_mode) {
            case 0: GRG_CUDA_TRY(launch_k(pdl, s, grid, kWarpRowThreads, level_warp_kernel<T, V, 0>, la)); break;
            case 1: GRG_CUDA_TRY(launch_k(pdl, s, grid, kWarpRowThreads, level_warp_kernel<T, V, 1>, la)); break;
            case 2: GRG_CUDA_TRY(launch_k(pdl, s, grid, kWarpRowThreads, level_warp_kernel<T, V, 2>, la)); break;
            default: GRG_CUDA_TRY(launch_k(pdl, s, grid, kWarpRowThreads, level_warp_kernel<T, V, 3>, la)); break;
        }
        GRG_LAUNCH_CHECK("level_warp_kernel");
    } else if (la.num_heavy > 0) {
        const dim3 grid(static_cast<unsigned>(la.num_heavy));
#define GRG_WIDE(INIT)                                                                            \
    if (exact) level_wide_kernel<T, V, INIT, true><<<grid, kWideThreads, 0, s>>>(la);            \
    else level_wide_kernel<T, V, INIT, false><<<grid, kWideThreads, 0, s>>>(la);
        switch (init_mode) {
            case 0: GRG_WIDE(0) break;
            case 1: GRG_WIDE(1) break;
            case 2: GRG_WIDE(2) break;
            default: GRG_WIDE(3) break;
        }
#undef GRG_WIDE
        GRG_LAUNCH_CHECK("level_wide_kernel");
    }
    return GRG_B200_OK;
}

template <int VM>
int launch_level_mx_typed(const LevelArgs& la, int init_mode, cudaStream_t s) {
    const int64_t narrow = la.num_rows - la.num_heavy;  // heavy positions form the suffix
    if (narrow > 0) {
        const int64_t warps = (narrow + (32 >> la.log2g) - 1) >> (5 - la.log2g);
        const dim3 grid(static_cast<unsigned>((warps + kNarrowWarps - 1) / kNarrowWarps));
        switch (init_mode) {
            case 0: level_mx_kernel<0, VM><<<grid, kNarrowThreads, 0, s>>>(la); break;
            case 1: level_mx_kernel<1, VM><<<grid, kNarrowThreads, 0, s>>>(la); break;
            case 2: level_mx_kernel<2, VM><<<grid, kNarrowThreads, 0, s>>>(la); break;
            default: level_mx_kernel<3, VM><<<grid, kNarrowThreads, 0, s>>>(la); break;
        }
        GRG_LAUNCH_CHECK("level_mx_kernel");
    }
    if (la.num_heavy > 0) {
        constexpr int rows_per_cta = kWarpRowThreads / 32;
        const dim3 grid(static_cast<unsigned>((la.num_heavy + rows_per_cta - 1) / rows_per_cta));
        switch (init_mode) {
            case 0: level_mx_warp_kernel<0, VM><<<grid, kWarpRowThreads, 0, s>>>(la); break;
            case 1: level_mx_warp_kernel<1, VM><<<grid, kWarpRowThreads, 0, s>>>(la); break;
            case 2: level_mx_warp_kernel<2, VM><<<grid, kWarpRowThreads, 0, s>>>(la); break;
            default: level_mx_warp_kernel<3, VM><<<grid, kWarpRowThreads, 0, s>>>(la); break;
        }
        GRG_LAUNCH_CHECK("level_mx_warp_kernel");
    }
    return GRG_B200_OK;
}

// Mixed level launches: narrow_variant 7 walks rows with 2 columns per lane, others with 4.
int launch_level_mx(LevelArgs la, int init_mode, int variant, cudaStream_t s) {
    const int vm = variant == 7 || variant >= 11 ? 2 : 4;
    const int64_t cols = (la.k + vm - 1) / vm;
    int log2g = 0;
    while ((1 << log2g) < cols && log2g < 5) ++log2g;
    la.log2g = log2g;
    return vm == 2 ? launch_level_mx_typed<2>(la, init_mode, s) : launch_level_mx_typed<4>(la, init_mode, s);
}

template <typename F>
int dispatch(const grg_b200_traverse_args* a, const Shape& sh, F&& f) {
    if (a->dtype == GRG_B200_F64) {
        if (sh.vec == 2) return f(double{}, std::integral_constant<int, 2>{});
        return f(double{}, std::integral_constant<int, 1>{});
    }
    if (sh.vec == 4) return f(float{}, std::integral_constant<int, 4>{});
    if (sh.vec == 2) return f(float{}, std::integral_constant<int, 2>{});
    return f(float{}, std::integral_constant<int, 1>{});
}

// Checked launch parameters of one non-empty level whose lists are at `blob` (run_level and
// the fused runs share them).
int build_level_args(const grg_b200_traverse_args* a, const Shape& sh, const grg_b200_level* L, const void* blob, LevelArgs& out) {
    if (!blob) return fail(GRG_B200_ERR_INVALID, "level blob is NULL");
    if (L->row_begin < 0 || L->row_begin + L->num_rows > a->num_nodes)
        return fail(GRG_B200_ERR_INVALID, "level rows [%lld, %lld) outside the %lld nodes", (long long)L->row_begin,
                    (long long)(L->row_begin + L->num_rows), (long long)a->num_nodes);
    const char* base = static_cast<const char*>(blob);
    LevelArgs la = level_args(a, sh);
    la.row_begin = L->row_begin;
    la.num_rows = L->num_rows;
    la.row_ptr = reinterpret_cast<const int32_t*>(base + L->off_row_ptr);
    la.entries = reinterpret_cast<const uint32_t*>(base + L->off_entries);
    la.heavy_rows = reinterpret_cast<const int32_t*>(base + L->off_heavy);
    la.row_ids = L->off_row_ids >= 0 ? reinterpret_cast<const int32_t*>(base + L->off_row_ids) : nullptr;
    if (L->list_align != 1 && L->list_align != 4) return fail(GRG_B200_ERR_INVALID, "list_align must be 1 or 4, got %d", L->list_align);
    if ((a->narrow_variant >= 6 || a->dtype == GRG_B200_MIXED) && L->list_align != 4)
        return fail(GRG_B200_ERR_INVALID, "narrow_variants 6/7 and mixed storage need padded gather lists (list_align 4)");
    if (L->list_align == 4 && (L->off_entries % 16) != 0) return fail(GRG_B200_ERR_INVALID, "padded lists must start 16-byte aligned");
    la.list_align = L->list_align;
    la.num_heavy = L->num_heavy;
    if (L->short_rows < 0 || L->short_rows > L->num_rows - L->num_heavy)
        return fail(GRG_B200_ERR_INVALID, "short_rows %lld outside [0, %lld]", (long long)L->short_rows,
                    (long long)(L->num_rows - L->num_heavy));
    la.short_rows = L->short_rows;
    la.num_slot_buckets = 0;
    if (L->num_slot_buckets < 0 || L->num_slot_buckets > GRG_B200_MAX_SLOT_BUCKETS)
        return fail(GRG_B200_ERR_INVALID, "num_slot_buckets %d outside [0, %d]", L->num_slot_buckets, GRG_B200_MAX_SLOT_BUCKETS);
    if (L->num_slot_buckets > 0) {
        if (L->list_align != 4 || L->slot_pos[0] != 0) return fail(GRG_B200_ERR_INVALID, "slot table needs padded lists starting at position 0");
        for (int b = 0; b < L->num_slot_buckets; ++b) {
            const int64_t end = b + 1 < L->num_slot_buckets ? L->slot_pos[b + 1] : L->num_rows - L->num_heavy;
            if (L->slot_width[b] < 0 || end < L->slot_pos[b] || L->slot_entry[b] < 0 || (L->slot_entry[b] & 3) ||
                L->slot_entry[b] + (end - L->slot_pos[b]) * 4 * L->slot_width[b] > L->num_entries)
                return fail(GRG_B200_ERR_INVALID, "slot bucket %d outside the level's lists", b);
            la.slot_pos[b] = L->slot_pos[b];
            la.slot_entry[b] = L->slot_entry[b];
            la.slot_width[b] = L->slot_width[b];
        }
        la.num_slot_buckets = L->num_slot_buckets;
    }
    la.log2s = 0;
    if (a->exact_order == 0 && a->narrow_variant >= 6 && a->dtype != GRG_B200_MIXED) {
        if (a->narrow_split >= 0) {
            la.log2s = a->narrow_split;
        } else {  // split long rows while the level alone would not fill the GPU twice over
            const int64_t narrow_rows = L->num_rows - L->num_heavy;
            const int64_t quads = narrow_rows > 0 ? (L->num_entries / 4) / narrow_rows : 0;
            const int64_t target_warps = 148 * 48 * 2;
            while (la.log2s < 3 && sh.log2g + la.log2s < 5 && (int64_t{2} << la.log2s) <= quads &&
                   ((narrow_rows << (sh.log2g + la.log2s + 1)) >> 5) <= target_warps)
                ++la.log2s;
        }
        if (sh.log2g + la.log2s > 5) la.log2s = 5 - sh.log2g;
    }
    la.heavy_threshold = L->num_heavy > 0 ? L->heavy_threshold : INT32_MAX;
    out = la;
    return GRG_B200_OK;
}

int run_level(const grg_b200_traverse_args* a, const Shape& sh, const grg_b200_level* L, const void* blob, cudaStream_t s) {
    if (L->num_rows < 0 || L->num_heavy < 0 || L->num_entries < 0)
        return fail(GRG_B200_ERR_INVALID, "negative level sizes");
    if (L->num_rows == 0) return GRG_B200_OK;
    LevelArgs la;
    const int rc = build_level_args(a, sh, L, blob, la);
    if (rc) return rc;
    const bool exact = a->exact_order != 0;
    if (a->dtype == GRG_B200_MIXED) return launch_level_mx(la, a->init_mode, a->narrow_variant, s);
    return dispatch(a, sh, [&](auto t, auto v) {
        return launch_level_typed<decltype(t), decltype(v)::value>(la, a->init_mode, exact, a->narrow_variant, a->heavy_variant,
                                                                   a->persist_ctas, (a->launch_flags & GRG_B200_LAUNCH_PDL) != 0, s);
    });
}

// Whether level L may join a fused run: resident, non-empty, at most fuse_entries entries,
// and a shape the run kernel reproduces bit for bit (default mode, padded lists, heavy rows one
// warp each, no row split).  `la` receives the level's launch parameters.
bool run_eligible(const grg_b200_traverse_args* a, const Shape& sh, const grg_b200_level& L, LevelArgs& la) {
    if (a->fuse_entries <= 0 || a->exact_order || a->dtype == GRG_B200_MIXED || a->heavy_variant != 2) return false;
    if (a->narrow_variant < 6 || a->narrow_variant == 8 || a->narrow_variant >= 12 || !a->dataflow_sync) return false;
    if (L.ring_slot >= 0 || L.num_rows <= 0 || L.num_entries > a->fuse_entries || L.list_align != 4) return false;
    if (L.num_heavy < 0 || L.num_heavy > L.num_rows || L.num_rows >= (int64_t{1} << 30)) return false;
    if (build_level_args(a, sh, &L, L.blob, la) != GRG_B200_OK) return false;
    return la.log2s == 0;
}

template <typename T, int V>
int launch_run_typed(RunArgs& p, int init_mode, int64_t max_blocks, cudaStream_t s) {
    int device = 0, sms = 0, per_sm = 0;
    GRG_CUDA_TRY(cudaGetDevice(&device));
    GRG_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    void (*kernel)(const RunArgs) = nullptr;
    switch (init_mode) {
        case 0: kernel = level_run_kernel<T, V, 0, 5>; break;
        case 1: kernel = level_run_kernel<T, V, 1, 5>; break;
        case 2: kernel = level_run_kernel<T, V, 2, 5>; break;
        default: kernel = level_run_kernel<T, V, 3, 5>; break;
    }
    GRG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kNarrowThreads, 0));
    if (per_sm < 1) return fail(GRG_B200_ERR_UNSUPPORTED, "the fused level run kernel does not fit on an SM");
    const int64_t resident = static_cast<int64_t>(sms) * per_sm;
    const int64_t grid = max_blocks < resident ? max_blocks : resident;
    // arrivals and the abort flag restart at zero; a timeout status in sync[2] stays for the host
    GRG_CUDA_TRY(cudaMemsetAsync(p.sync, 0, 2 * sizeof(int32_t), s));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(grid));
    cfg.blockDim = dim3(kNarrowThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;  // every CTA resident: the grid barrier can complete
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    GRG_CUDA_TRY(cudaLaunchKernelEx(&cfg, kernel, p));
    GRG_LAUNCH_CHECK("level_run_kernel");
    return GRG_B200_OK;
}

// Runs levels [first, first + count) (all run_eligible, launch parameters in `las`) as one
// cooperative launch.
int launch_run(const grg_b200_traverse_args* a, const Shape& sh, const LevelArgs* las, int count, cudaStream_t s) {
    if (count < 1 || count > kRunMaxLevels) return fail(GRG_B200_ERR_INVALID, "fused run of %d levels", count);
    static thread_local RunArgs p;  // about 20 KB: kept off the stack
    std::memset(&p, 0, sizeof(p));
    p.sync = static_cast<int32_t*>(a->dataflow_sync);
    p.num_levels = count;
    int64_t max_blocks = 1;
    for (int i = 0; i < count; ++i) {
        const LevelArgs& la = las[i];
        const int64_t narrow = la.num_rows - la.num_heavy;
        constexpr int rows_per_cta = kWarpRowThreads / 32;
        const int64_t heavy_blocks = (la.num_heavy + rows_per_cta - 1) / rows_per_cta;
        const int64_t warps = (narrow + (32 >> la.log2g) - 1) >> (5 - la.log2g);
        p.lv[i] = la;
        p.heavy_blocks[i] = heavy_blocks;
        p.blocks[i] = heavy_blocks + (warps + kNarrowWarps - 1) / kNarrowWarps;
        if (p.blocks[i] > max_blocks) max_blocks = p.blocks[i];
    }
    return dispatch(a, sh, [&](auto t, auto v) { return launch_run_typed<decltype(t), decltype(v)::value>(p, a->init_mode, max_blocks, s); });
}

int seed_up_impl(const grg_b200_traverse_args* a, const Shape& sh, cudaStream_t s) {
    const bool pdl = (a->launch_flags & GRG_B200_LAUNCH_PDL) != 0;
    if (a->level0_rows <= 0) return GRG_B200_OK;
    if (!a->input) return fail(GRG_B200_ERR_INVALID, "input is NULL");
    if (a->by_individual && !a->sample_to_individual) return fail(GRG_B200_ERR_INVALID, "sample_to_individual is NULL");
    LevelArgs la = level_args(a, sh);
    la.row_begin = 0;
    la.num_rows = a->level0_rows;
    const dim3 grid = grid_for(la.num_rows, la.log2g, 256);
    if (a->dtype == GRG_B200_MIXED) {
        switch (a->init_mode) {
            case 0: seed_up_mx_kernel<0><<<grid, 256, 0, s>>>(la, a->num_samples, a->sample_to_individual, a->by_individual); break;
            case 1: seed_up_mx_kernel<1><<<grid, 256, 0, s>>>(la, a->num_samples, a->sample_to_individual, a->by_individual); break;
            case 2: seed_up_mx_kernel<2><<<grid, 256, 0, s>>>(la, a->num_samples, a->sample_to_individual, a->by_individual); break;
            default: seed_up_mx_kernel<3><<<grid, 256, 0, s>>>(la, a->num_samples, a->sample_to_individual, a->by_individual); break;
        }
        GRG_LAUNCH_CHECK("seed_up_mx_kernel");
        return (int)GRG_B200_OK;
    }
    return dispatch(a, sh, [&](auto t, auto v) {
        using T = decltype(t);
        constexpr int V = decltype(v)::value;
        switch (a->init_mode) {
            case 0: GRG_CUDA_TRY(launch_k(pdl, s, grid, 256, seed_up_kernel<T, V, 0>, la, a->num_samples, a->sample_to_individual, a->by_individual)); break;
            case 1: GRG_CUDA_TRY(launch_k(pdl, s, grid, 256, seed_up_kernel<T, V, 1>, la, a->num_samples, a->sample_to_individual, a->by_individual)); break;
            case 2: GRG_CUDA_TRY(launch_k(pdl, s, grid, 256, seed_up_kernel<T, V, 2>, la, a->num_samples, a->sample_to_individual, a->by_individual)); break;
            default: GRG_CUDA_TRY(launch_k(pdl, s, grid, 256, seed_up_kernel<T, V, 3>, la, a->num_samples, a->sample_to_individual, a->by_individual)); break;
        }
        GRG_LAUNCH_CHECK("seed_up_kernel");
        return (int)GRG_B200_OK;
    });
}

OutArgs out_args(const grg_b200_traverse_args* a, const Shape& sh) {
    OutArgs o{};
    o.state = a->state;
    o.ld_state = a->ld_state;
    o.out = a->output;
    o.ld_out = a->ld_output;
    o.bias = a->endpoint_bias;
    o.init_vector = a->init_vector;
    o.bias_mode = a->emit_all_nodes ? GRG_B200_BIAS_NONE : a->bias_mode;
    o.k = a->k;
    o.log2g = sh.log2g;
    o.err = a->error_word;
    o.lim = a->num_nodes;
    if (a->dtype == GRG_B200_MIXED)
        o.state_lo = static_cast<const char*>(a->state) + GRG_B200_MIX_PLANE(a->num_nodes * a->ld_state * 4);
    return o;
}

int output_up_impl(const grg_b200_traverse_args* a, const Shape& sh, cudaStream_t s) {
    const bool pdl = (a->launch_flags & GRG_B200_LAUNCH_PDL) != 0;
    if (!a->output || !a->sel_mut_ptr || (!a->sel_mut_idx && a->num_mutations > 0))
        return fail(GRG_B200_ERR_INVALID, "up output needs output and sel_mut");
    if (a->use_miss && (!a->miss || !a->sel_miss_ptr)) return fail(GRG_B200_ERR_INVALID, "up miss output needs miss and sel_miss");
    if (a->num_mutations == 0) return GRG_B200_OK;
    OutArgs o = out_args(a, sh);
    o.rows = a->num_mutations;
    o.ptr = a->sel_mut_ptr;
    o.idx = a->sel_mut_idx;
    const dim3 grid = grid_for(o.rows, o.log2g, 256);
    if (a->dtype == GRG_B200_MIXED) {
        gather_out_mx_kernel<false><<<grid, 256, 0, s>>>(o);
        GRG_LAUNCH_CHECK("gather_out_mx_kernel(sel_mut)");
        if (a->use_miss) {
            OutArgs m = o;
            m.ptr = a->sel_miss_ptr;
            m.idx = a->sel_miss_idx;
            m.out = a->miss;
            m.ld_out = a->ld_miss;
            m.bias_mode = GRG_B200_BIAS_NONE;
            gather_out_mx_kernel<false><<<grid, 256, 0, s>>>(m);
            GRG_LAUNCH_CHECK("gather_out_mx_kernel(sel_miss)");
        }
        return (int)GRG_B200_OK;
    }
    return dispatch(a, sh, [&](auto t, auto v) {
        using T = decltype(t);
        constexpr int V = decltype(v)::value;
        GRG_CUDA_TRY(launch_k(pdl, s, grid, 256, gather_out_kernel<T, V, false>, o));
        GRG_LAUNCH_CHECK("gather_out_kernel(sel_mut)");
        if (a->use_miss) {
            OutArgs m = o;
            m.ptr = a->sel_miss_ptr;
            m.idx = a->sel_miss_idx;
            m.out = a->miss;
            m.ld_out = a->ld_miss;
            m.bias_mode = GRG_B200_BIAS_NONE;
            GRG_CUDA_TRY(launch_k(pdl, s, grid, 256, gather_out_kernel<T, V, false>, m));
            GRG_LAUNCH_CHECK("gather_out_kernel(sel_miss)");
        }
        return (int)GRG_B200_OK;
    });
}

int output_down_impl(const grg_b200_traverse_args* a, const Shape& sh, cudaStream_t s) {
    const bool pdl = (a->launch_flags & GRG_B200_LAUNCH_PDL) != 0;
    if (!a->output) return fail(GRG_B200_ERR_INVALID, "output is NULL");
    OutArgs o = out_args(a, sh);
    if (a->by_individual) {
        if (!a->ind_ptr || !a->ind_samples) return fail(GRG_B200_ERR_INVALID, "by_individual needs ind_ptr/ind_samples");
        o.rows = a->num_individuals;
        o.ptr = a->ind_ptr;
        o.idx = a->ind_samples;
        o.lim = a->num_samples;
    } else {
        o.rows = a->num_samples;
    }
    if (o.rows == 0) return GRG_B200_OK;
    const dim3 grid = grid_for(o.rows, o.log2g, 256);
    if (a->dtype == GRG_B200_MIXED) {
        if (a->by_individual) gather_out_mx_kernel<true><<<grid, 256, 0, s>>>(o);
        else copy_out_mx_kernel<<<grid, 256, 0, s>>>(o);
        GRG_LAUNCH_CHECK("output_down_mx");
        return (int)GRG_B200_OK;
    }
    return dispatch(a, sh, [&](auto t, auto v) {
        using T = decltype(t);
        constexpr int V = decltype(v)::value;
        if (a->by_individual) GRG_CUDA_TRY(launch_k(pdl, s, grid, 256, gather_out_kernel<T, V, true>, o));
        else GRG_CUDA_TRY(launch_k(pdl, s, grid, 256, copy_out_kernel<T, V>, o));
        GRG_LAUNCH_CHECK("output_down");
        return (int)GRG_B200_OK;
    });
}

int emit_all_impl(const grg_b200_traverse_args* a, const Shape& sh, cudaStream_t s) {
    const bool pdl = (a->launch_flags & GRG_B200_LAUNCH_PDL) != 0;
    if (!a->output || !a->inv_node_perm) return fail(GRG_B200_ERR_INVALID, "emit_all_nodes needs output and inv_node_perm");
    OutArgs o = out_args(a, sh);
    o.rows = a->num_nodes;
    o.idx = a->inv_node_perm;
    const dim3 grid = grid_for(o.rows, o.log2g, 256);
    if (a->dtype == GRG_B200_MIXED) {
        emit_all_mx_kernel<<<grid, 256, 0, s>>>(o);
        GRG_LAUNCH_CHECK("emit_all_mx_kernel");
        return (int)GRG_B200_OK;
    }
    return dispatch(a, sh, [&](auto t, auto v) {
        using T = decltype(t);
        constexpr int V = decltype(v)::value;
        GRG_CUDA_TRY(launch_k(pdl, s, grid, 256, emit_all_kernel<T, V>, o));
        GRG_LAUNCH_CHECK("emit_all_kernel");
        return (int)GRG_B200_OK;
    });
}

// Dataflow schedule: eligible when every level is resident with padded lists, the default
// (fast) mode and a plain dtype; otherwise the traversal runs level by level.
bool dataflow_eligible(const grg_b200_traverse_args* a) {
    if (a->schedule != GRG_B200_SCHEDULE_DATAFLOW || !a->dataflow_sync) return false;
    if (a->exact_order || a->dtype == GRG_B200_MIXED || a->num_levels > kDfMaxLevels) return false;
    for (int i = 0; i < a->num_levels; ++i) {
        const grg_b200_level& L = a->levels[i];
        if (L.ring_slot >= 0 || L.list_align != 4 || L.num_rows >= INT32_MAX) return false;
    }
    return true;
}

template <typename T, int V>
int launch_dataflow_typed(DfArgs& p, int init_mode, cudaStream_t s) {
    int device = 0, sms = 0, per_sm = 0;
    GRG_CUDA_TRY(cudaGetDevice(&device));
    GRG_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
#define GRG_DF(INIT)                                                                                      \
    GRG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dataflow_kernel<T, V, INIT>, kDfThreads, 0)); \
    dataflow_kernel<T, V, INIT><<<dim3(static_cast<unsigned>(sms * (per_sm > 0 ? per_sm : 1))), kDfThreads, 0, s>>>(p);
    switch (init_mode) {
        case 0: GRG_DF(0) break;
        case 1: GRG_DF(1) break;
        case 2: GRG_DF(2) break;
        default: GRG_DF(3) break;
    }
#undef GRG_DF
    GRG_LAUNCH_CHECK("dataflow_kernel");
    return GRG_B200_OK;
}

int run_dataflow(const grg_b200_traverse_args* a, const Shape& sh, cudaStream_t s) {
    DfArgs p;  // launch parameters (about 6 KB, copied into the launch)
    std::memset(&p, 0, sizeof(p));
    p.a = level_args(a, sh);
    p.a.log2s = 0;
    p.sync = static_cast<int32_t*>(a->dataflow_sync);
    p.num_levels = a->num_levels;
    int64_t tasks = 0, fill_begin = INT64_MAX, fill_end = 0;
    const int rows_per_warp_log2 = 5 - sh.log2g;
    for (int i = 0; i < a->num_levels; ++i) {
        const grg_b200_level& L = a->levels[i];
        const char* base = static_cast<const char*>(L.blob);
        if (L.num_rows > 0 && !base) return fail(GRG_B200_ERR_INVALID, "level blob is NULL");
        if (L.row_begin < 0 || L.row_begin + L.num_rows > a->num_nodes)
            return fail(GRG_B200_ERR_INVALID, "level rows outside the %lld nodes", (long long)a->num_nodes);
        if (L.list_align == 4 && (L.off_entries % 16) != 0) return fail(GRG_B200_ERR_INVALID, "padded lists must start 16-byte aligned");
        DfLevel& d = p.lv[i];
        d.row_ptr = reinterpret_cast<const int32_t*>(base + L.off_row_ptr);
        d.codes = reinterpret_cast<const uint4*>(base + L.off_entries);
        d.row_ids = L.off_row_ids >= 0 ? reinterpret_cast<const int32_t*>(base + L.off_row_ids) : nullptr;
        d.row_begin = L.row_begin;
        d.num_rows = static_cast<int32_t>(L.num_rows);
        d.num_heavy = static_cast<int32_t>(L.num_heavy);
        p.task_begin[i] = static_cast<int32_t>(tasks);
        const int64_t narrow = L.num_rows - L.num_heavy;
        tasks += L.num_heavy + ((narrow + (int64_t{1} << rows_per_warp_log2) - 1) >> rows_per_warp_log2);
        if (L.num_rows > 0) {
            fill_begin = L.row_begin < fill_begin ? L.row_begin : fill_begin;
            fill_end = L.row_begin + L.num_rows > fill_end ? L.row_begin + L.num_rows : fill_end;
        }
    }
    if (tasks >= INT32_MAX) return fail(GRG_B200_ERR_UNSUPPORTED, "dataflow schedule: too many tasks");
    p.task_begin[a->num_levels] = static_cast<int32_t>(tasks);
    p.total_tasks = static_cast<int32_t>(tasks);
    GRG_CUDA_TRY(cudaMemsetAsync(a->dataflow_sync, 0, 4 * sizeof(int32_t), s));
    if (fill_end > fill_begin) {
        const int64_t n = (fill_end - fill_begin) * a->ld_state;
        const int64_t blocks = (n + 255) / 256 < 148 * 32 ? (n + 255) / 256 : 148 * 32;
        if (a->dtype == GRG_B200_F64)
            sentinel_fill_kernel<double><<<static_cast<unsigned>(blocks), 256, 0, s>>>(static_cast<double*>(a->state) + fill_begin * a->ld_state, n);
        else
            sentinel_fill_kernel<float><<<static_cast<unsigned>(blocks), 256, 0, s>>>(static_cast<float*>(a->state) + fill_begin * a->ld_state, n);
        GRG_LAUNCH_CHECK("sentinel_fill_kernel");
    }
    if (a->direction == GRG_B200_UP) {
        const int rc = seed_up_impl(a, sh, s);
        if (rc) return rc;
    }
    if (tasks == 0) return GRG_B200_OK;
    return dispatch(a, sh, [&](auto t, auto v) { return launch_dataflow_typed<decltype(t), decltype(v)::value>(p, a->init_mode, s); });
}

// Mixed down: encoded copies of the input (and miss) rows, which the level lists read.
int encode_down_inputs(const grg_b200_traverse_args* a, const Shape& sh, cudaStream_t s) {
    if (a->num_mutations == 0) return GRG_B200_OK;
    const LevelArgs la = level_args(a, sh);
    const int64_t ld = a->ld_state;
    int log2g = 0;
    while ((1 << log2g) < (ld + 3) / 4 && log2g < 5) ++log2g;
    const dim3 grid = grid_for(a->num_mutations, log2g, 256);
    mx_encode_rows_kernel<<<grid, 256, 0, s>>>(static_cast<const double*>(a->input), a->ld_input, a->num_mutations, a->k,
                                               static_cast<float*>(const_cast<void*>(la.x)),
                                               static_cast<short*>(const_cast<void*>(la.x_lo)), ld, log2g);
    GRG_LAUNCH_CHECK("mx_encode_rows_kernel(input)");
    if (a->use_miss) {
        mx_encode_rows_kernel<<<grid, 256, 0, s>>>(static_cast<const double*>(a->miss), a->ld_miss, a->num_mutations, a->k,
                                                   static_cast<float*>(const_cast<void*>(la.miss)),
                                                   static_cast<short*>(const_cast<void*>(la.miss_lo)), ld, log2g);
        GRG_LAUNCH_CHECK("mx_encode_rows_kernel(miss)");
    }
    return GRG_B200_OK;
}

}  // namespace

// ---------------------------------------------------------------------------------------
// Standardised-operator row step (grg_b200_rowop): one pass over a [rows, k] buffer applying
// the per-row affine map of the header, with deterministic column sums.  A block owns
// GRG_B200_ROWOP_ROWS_PER_BLOCK consecutive rows; its 256 threads form ny = 256 / kt row
// groups of kt column lanes (kt: k rounded up to a power of two, at most 256).  Lane (x, y)
// walks rows y, y + ny, ... of the block for column c0 + x, so a warp reads contiguous
// columns of a row; the ny partial sums are added in y order, and the finalize kernel adds
// the blocks' partials in block order.
// ---------------------------------------------------------------------------------------
constexpr int kRowopThreads = 256;

__global__ void __launch_bounds__(kRowopThreads) rowop_kernel(grg_b200_rowop_args a, int log2kt, int64_t rows_per_block) {
    __shared__ double red[kRowopThreads];
    const int kt = 1 << log2kt;
    const int tx = threadIdx.x & (kt - 1);
    const int ty = threadIdx.x >> log2kt;
    const int ny = kRowopThreads >> log2kt;
    const int64_t r0 = static_cast<int64_t>(blockIdx.x) * rows_per_block;
    const int64_t r1 = r0 + rows_per_block < a.rows ? r0 + rows_per_block : a.rows;
    for (int64_t c0 = 0; c0 < a.k; c0 += kt) {
        const int64_t j = c0 + tx;
        const bool active = j < a.k;
        const double cs = active && a.col_sub ? __ldg(a.col_sub + j) : 0.0;
        double part = 0.0;
        if (active) {
            for (int64_t r = r0 + ty; r < r1; r += ny) {
                const int64_t e = r * a.ld + j;
                double t = __ldg(a.src + e);
                if (a.miss_in) t = __dadd_rn(t, __dmul_rn(__ldg(a.miss_in + e), __ldg(a.miss_scale + r)));
                if (a.pre_scale) t = __dmul_rn(t, __ldg(a.pre_scale + r));
                if (a.col_sub) t = __dsub_rn(t, a.sub_scale ? __dmul_rn(cs, __ldg(a.sub_scale + r)) : cs);
                if (a.post_scale) t = __dmul_rn(t, __ldg(a.post_scale + r));
                a.dst[e] = t;
                if (a.miss_out) a.miss_out[e] = __dmul_rn(t, __ldg(a.miss_out_scale + r));
                if (a.col_sums) part = __dadd_rn(part, a.sum_weight ? __dmul_rn(t, __ldg(a.sum_weight + r)) : t);
            }
        }
        if (a.col_sums) {  // uniform across the block
            red[threadIdx.x] = part;
            __syncthreads();
            if (ty == 0 && active) {
                double s = red[tx];
                for (int y = 1; y < ny; ++y) s = __dadd_rn(s, red[(y << log2kt) + tx]);
                a.partials[static_cast<int64_t>(blockIdx.x) * a.k + j] = s;
            }
            __syncthreads();
        }
    }
}

// One CTA per column: thread t adds the partials of blocks t, t + 256, ... in order, then a
// fixed tree combines the 256 sums.
__global__ void __launch_bounds__(256) rowop_finalize_kernel(const double* partials, int64_t blocks, int64_t k, double* sums) {
    __shared__ double red[256];
    const int64_t j = blockIdx.x;
    double s = 0.0;
    for (int64_t b = threadIdx.x; b < blocks; b += 256) s = __dadd_rn(s, partials[b * k + j]);
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (static_cast<int>(threadIdx.x) < w) red[threadIdx.x] = __dadd_rn(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[j] = red[0];
}

struct grg_b200_ring {
    int device;
    int num_slots;
    cudaStream_t copy;
    cudaEvent_t fork;
    cudaEvent_t join;
    cudaEvent_t* ready;
    cudaEvent_t* free_ev;
};

extern "C" {

int grg_b200_abi_version(void) { return GRG_B200_ABI_VERSION; }

int grg_b200_rowop(const grg_b200_rowop_args* a, void* stream_handle) {
    if (!a) return fail(GRG_B200_ERR_INVALID, "args is NULL");
    if (a->rows < 0 || a->k < 1 || a->ld < a->k)
        return fail(GRG_B200_ERR_INVALID, "rowop needs rows >= 0, k >= 1 and ld >= k (got %lld, %lld, %lld)",
                    (long long)a->rows, (long long)a->k, (long long)a->ld);
    if (!a->src || !a->dst) return fail(GRG_B200_ERR_INVALID, "rowop src/dst is NULL");
    if (a->miss_in && !a->miss_scale) return fail(GRG_B200_ERR_INVALID, "rowop miss_in needs miss_scale");
    if (a->miss_out && !a->miss_out_scale) return fail(GRG_B200_ERR_INVALID, "rowop miss_out needs miss_out_scale");
    if (a->col_sums && (!a->partials || !a->sums)) return fail(GRG_B200_ERR_INVALID, "rowop col_sums needs partials and sums");
    if (a->rows == 0) return GRG_B200_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream_handle);
    int log2kt = 0;
    while ((int64_t{1} << log2kt) < a->k && log2kt < 8) ++log2kt;
    const int64_t blocks = GRG_B200_ROWOP_BLOCKS(a->rows);
    const int64_t rows_per_block = (a->rows + blocks - 1) / blocks;
    if (a->k > 0x7fffffff) return fail(GRG_B200_ERR_UNSUPPORTED, "rowop: k = %lld is too large", (long long)a->k);
    rowop_kernel<<<dim3(static_cast<unsigned>(blocks)), kRowopThreads, 0, s>>>(*a, log2kt, rows_per_block);
    GRG_LAUNCH_CHECK("rowop_kernel");
    if (a->col_sums) {
        rowop_finalize_kernel<<<dim3(static_cast<unsigned>(a->k)), 256, 0, s>>>(a->partials, blocks, a->k, a->sums);
        GRG_LAUNCH_CHECK("rowop_finalize_kernel");
    }
    return GRG_B200_OK;
}


size_t grg_b200_last_error(char* buf, size_t buf_size) {
    const size_t n = strlen(g_last_error);
    if (buf && buf_size) {
        const size_t m = n < buf_size - 1 ? n : buf_size - 1;
        memcpy(buf, g_last_error, m);
        buf[m] = '\0';
    }
    return n;
}

int grg_b200_ring_create(int device, int num_slots, grg_b200_ring** out) {
    if (!out || num_slots < 1) return fail(GRG_B200_ERR_INVALID, "ring needs num_slots >= 1 and an out pointer");
    *out = nullptr;
    int prev = 0;
    GRG_CUDA_TRY(cudaGetDevice(&prev));
    GRG_CUDA_TRY(cudaSetDevice(device));
    grg_b200_ring* r = new grg_b200_ring{};
    r->device = device;
    r->num_slots = num_slots;
    r->ready = new cudaEvent_t[num_slots]();
    r->free_ev = new cudaEvent_t[num_slots]();
    cudaError_t e = cudaStreamCreateWithFlags(&r->copy, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->join, cudaEventDisableTiming);
    for (int i = 0; i < num_slots && e == cudaSuccess; ++i) {
        e = cudaEventCreateWithFlags(&r->ready[i], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->free_ev[i], cudaEventDisableTiming);
    }
    cudaSetDevice(prev);
    if (e != cudaSuccess) {
        grg_b200_ring_destroy(r);
        return fail(GRG_B200_ERR_CUDA, "ring creation failed: %s", cudaGetErrorString(e));
    }
    *out = r;
    return GRG_B200_OK;
}

int grg_b200_ring_destroy(grg_b200_ring* r) {
    if (!r) return GRG_B200_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(r->device);
    if (r->copy) cudaStreamSynchronize(r->copy);
    for (int i = 0; i < r->num_slots; ++i) {
        if (r->ready && r->ready[i]) cudaEventDestroy(r->ready[i]);
        if (r->free_ev && r->free_ev[i]) cudaEventDestroy(r->free_ev[i]);
    }
    if (r->fork) cudaEventDestroy(r->fork);
    if (r->join) cudaEventDestroy(r->join);
    if (r->copy) cudaStreamDestroy(r->copy);
    cudaSetDevice(prev);
    delete[] r->ready;
    delete[] r->free_ev;
    delete r;
    return GRG_B200_OK;
}

int grg_b200_seed_up(const grg_b200_traverse_args* a, void* stream) {
    int rc = validate_common(a);
    if (rc) return rc;
    return seed_up_impl(a, choose_shape(a), static_cast<cudaStream_t>(stream));
}

int grg_b200_run_level(const grg_b200_traverse_args* a, const grg_b200_level* level, void* stream) {
    int rc = validate_common(a);
    if (rc) return rc;
    if (!level) return fail(GRG_B200_ERR_INVALID, "level is NULL");
    return run_level(a, choose_shape(a), level, level->blob, static_cast<cudaStream_t>(stream));
}

int grg_b200_output_up(const grg_b200_traverse_args* a, void* stream) {
    int rc = validate_common(a);
    if (rc) return rc;
    return output_up_impl(a, choose_shape(a), static_cast<cudaStream_t>(stream));
}

int grg_b200_output_down(const grg_b200_traverse_args* a, void* stream) {
    int rc = validate_common(a);
    if (rc) return rc;
    return output_down_impl(a, choose_shape(a), static_cast<cudaStream_t>(stream));
}

int grg_b200_emit_all(const grg_b200_traverse_args* a, void* stream) {
    int rc = validate_common(a);
    if (rc) return rc;
    return emit_all_impl(a, choose_shape(a), static_cast<cudaStream_t>(stream));
}

int grg_b200_traverse(const grg_b200_traverse_args* a, void* stream_handle) {
    int rc = validate_common(a);
    if (rc) return rc;
    if (a->num_levels < 0 || (a->num_levels > 0 && !a->levels)) return fail(GRG_B200_ERR_INVALID, "levels missing");
    if (a->direction == GRG_B200_DOWN && !a->input && a->num_mutations > 0) return fail(GRG_B200_ERR_INVALID, "input is NULL");
    if (a->direction == GRG_B200_DOWN && a->use_miss && !a->miss) return fail(GRG_B200_ERR_INVALID, "miss input is NULL");
    cudaStream_t s = static_cast<cudaStream_t>(stream_handle);
    const Shape sh = choose_shape(a);

    bool any_streamed = false;
    for (int i = 0; i < a->num_levels; ++i) {
        const grg_b200_level& L = a->levels[i];
        if (L.ring_slot >= 0) {
            any_streamed = true;
            if (!a->ring || L.ring_slot >= a->num_slots || L.ring_slot >= a->ring->num_slots || !a->slot_buffers || !a->slot_bytes)
                return fail(GRG_B200_ERR_INVALID, "level %d is streamed through slot %d but the ring is missing or too small", i, L.ring_slot);
            if (L.blob_bytes > a->slot_bytes[L.ring_slot])
                return fail(GRG_B200_ERR_INVALID, "level %d needs %lld bytes, slot %d has %lld", i, (long long)L.blob_bytes,
                            L.ring_slot, (long long)a->slot_bytes[L.ring_slot]);
        }
    }

    if (!any_streamed && dataflow_eligible(a)) {
        rc = run_dataflow(a, sh, s);
        if (rc) return rc;
        if (a->emit_all_nodes) return emit_all_impl(a, sh, s);
        if (a->direction == GRG_B200_UP) return output_up_impl(a, sh, s);
        return output_down_impl(a, sh, s);
    }
    grg_b200_traverse_args no_pdl;
    if (any_streamed && (a->launch_flags & GRG_B200_LAUNCH_PDL)) {  // ring copies sit between the level launches
        no_pdl = *a;
        no_pdl.launch_flags &= ~GRG_B200_LAUNCH_PDL;
        a = &no_pdl;
    }
    if (a->direction == GRG_B200_UP) {
        rc = seed_up_impl(a, sh, s);
        if (rc) return rc;
    } else if (a->dtype == GRG_B200_MIXED) {
        rc = encode_down_inputs(a, sh, s);
        if (rc) return rc;
    }
    // Fork the copy stream off the caller's stream so streamed copies are ordered after the
    // caller's earlier work (and join a CUDA graph capture in progress).
    bool used[256] = {false};
    if (any_streamed) {
        if (a->ring->num_slots > 256) return fail(GRG_B200_ERR_UNSUPPORTED, "at most 256 ring slots");
        GRG_CUDA_TRY(cudaEventRecord(a->ring->fork, s));
        GRG_CUDA_TRY(cudaStreamWaitEvent(a->ring->copy, a->ring->fork, 0));
    }
    for (int i = 0; i < a->num_levels; ++i) {
        if (a->fuse_entries > 0) {  // a run of small resident levels: one cooperative launch
            static thread_local LevelArgs run_las[kRunMaxLevels];
            int j = i, n = 0;
            while (j < a->num_levels && n < kRunMaxLevels) {
                if (a->levels[j].num_rows == 0) {  // an empty level launches nothing
                    ++j;
                    continue;
                }
                if (!run_eligible(a, sh, a->levels[j], run_las[n])) break;
                ++n;
                ++j;
            }
            if (n >= 2) {
                rc = launch_run(a, sh, run_las, n, s);
                if (rc) return rc;
                i = j - 1;
                continue;
            }
        }
        const grg_b200_level& L = a->levels[i];
        const void* blob = L.blob;
        if (L.ring_slot >= 0 && L.num_rows > 0) {
            grg_b200_ring* r = a->ring;
            if (used[L.ring_slot]) GRG_CUDA_TRY(cudaStreamWaitEvent(r->copy, r->free_ev[L.ring_slot], 0));
            GRG_CUDA_TRY(cudaMemcpyAsync(a->slot_buffers[L.ring_slot], L.blob, static_cast<size_t>(L.blob_bytes), cudaMemcpyHostToDevice, r->copy));
            GRG_CUDA_TRY(cudaEventRecord(r->ready[L.ring_slot], r->copy));
            GRG_CUDA_TRY(cudaStreamWaitEvent(s, r->ready[L.ring_slot], 0));
            blob = a->slot_buffers[L.ring_slot];
        }
        rc = run_level(a, sh, &L, blob, s);
        if (rc) return rc;
        if (L.ring_slot >= 0 && L.num_rows > 0) {
            GRG_CUDA_TRY(cudaEventRecord(a->ring->free_ev[L.ring_slot], s));
            used[L.ring_slot] = true;
        }
    }
    if (any_streamed) {
        GRG_CUDA_TRY(cudaEventRecord(a->ring->join, a->ring->copy));
        GRG_CUDA_TRY(cudaStreamWaitEvent(s, a->ring->join, 0));
    }
    if (a->emit_all_nodes) return emit_all_impl(a, sh, s);
    if (a->direction == GRG_B200_UP) return output_up_impl(a, sh, s);
    return output_down_impl(a, sh, s);
}

// ---------------------------------------------------------------------------------------
// Allocation-free traversal: the node state lives in a fixed device array of this library.
//
// Some callers cannot allocate device memory: C/FFI hosts with no device allocator of their
// own, plugins running inside another framework's memory manager, and code that must not
// allocate while a stream is being captured.  grg_b200_traverse_static serves them: it takes
// the same arguments as grg_b200_traverse (inputs, outputs and resident level blobs all come
// from the caller) but ignores args->state/ld_state and keeps the traversal's node state in
// g_static_state below.  That array holds GRG_B200_STATIC_STATE_BYTES on every GPU whose
// context loads this library, for the lifetime of the process.
// ---------------------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_static_state[GRG_B200_STATIC_STATE_BYTES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_static_mutex;
void* g_static_ptr[kMaxDevices] = {};
void* g_static_ctx[kMaxDevices] = {};  // the driver context each cached address belongs to

// The calling thread's current driver context (nullptr if none, or if the query is not
// available).  A module's device symbols have one address per context, so a cached address
// of g_static_state is valid only while the context it was taken in is current: after
// cudaDeviceReset, or when a host drives the device from a context it created itself, the
// context differs and the address is looked up again.
void* current_context() {
    using GetCurrentFn = int (*)(void**);
    static const GetCurrentFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<GetCurrentFn>(p);
    }();
    void* ctx = nullptr;
    if (!fn || fn(&ctx) != 0) return nullptr;
    return ctx;
}

// Device address of g_static_state on the current device, looked up once per device and
// context (the host symbol g_static_state is only a stand-in and must never reach a kernel).
int static_state_address(void** out) {
    int device = 0;
    GRG_CUDA_TRY(cudaGetDevice(&device));
    if (device < 0 || device >= kMaxDevices) return fail(GRG_B200_ERR_UNSUPPORTED, "device ordinal %d above %d", device, kMaxDevices);
    void* ctx = current_context();  // nullptr before the runtime has made a context current
    std::lock_guard<std::mutex> lock(g_static_mutex);
    if (!g_static_ptr[device] || !ctx || g_static_ctx[device] != ctx) {
        void* ptr = nullptr;
        const cudaError_t err = cudaGetSymbolAddress(&ptr, g_static_state);  // makes the context current
        if (err != cudaSuccess || !ptr)
            return fail(GRG_B200_ERR_CUDA, "cudaGetSymbolAddress(g_static_state) on device %d failed: %s", device,
                        cudaGetErrorString(err));
        g_static_ptr[device] = ptr;
        g_static_ctx[device] = current_context();
    }
    *out = g_static_ptr[device];
    return GRG_B200_OK;
}
}  // namespace

int grg_b200_traverse_static(const grg_b200_traverse_args* a, void* stream_handle) {
    if (!a) return fail(GRG_B200_ERR_INVALID, "args is NULL");
    if (a->k < 1) return fail(GRG_B200_ERR_INVALID, "k must be >= 1, got %lld", (long long)a->k);
    if (a->dtype == GRG_B200_MIXED) return fail(GRG_B200_ERR_UNSUPPORTED, "grg_b200_traverse_static serves the FP64 and FP32 dtypes only");
    const int64_t esize = a->dtype == GRG_B200_F64 ? 8 : 4;
    if (a->num_nodes < 0 || a->num_nodes > (int64_t)GRG_B200_STATIC_STATE_BYTES / esize / a->k)
        return fail(GRG_B200_ERR_UNSUPPORTED,
                    "grg_b200_traverse_static holds at most %lld bytes of node state; %lld nodes x k=%lld need %lld",
                    (long long)GRG_B200_STATIC_STATE_BYTES, (long long)a->num_nodes, (long long)a->k,
                    (long long)(a->num_nodes * a->k * esize));
    for (int i = 0; a->levels && i < a->num_levels; ++i)
        if (a->levels[i].ring_slot >= 0)
            return fail(GRG_B200_ERR_UNSUPPORTED, "grg_b200_traverse_static needs every level resident (level %d is streamed)", i);
    void* state = nullptr;
    const int rc = static_state_address(&state);
    if (rc) return rc;
    grg_b200_traverse_args local = *a;
    local.state = state;
    local.ld_state = a->k;
    local.ring = nullptr;
    local.slot_buffers = nullptr;
    local.slot_bytes = nullptr;
    local.num_slots = 0;
    return grg_b200_traverse(&local, stream_handle);
}

}  // extern "C"
