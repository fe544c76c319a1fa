// pg_common.cuh -- shared constants, device helpers and the workspace layout
// of the paragram_b200 diagram builder.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace pg
{

// Status codes of a cell, as in the reference (faster_convex_cell.cuh:99-108).
enum Status : int
{
    kSuccess = 0,
    kPlaneOverflow = 1,
    kVertexOverflow = 2,
    kEmptyCell = 3,
    kSecurityRadiusNotReached = 4,
    kInconsistentBoundary = 5,
};

constexpr int kMaxVertsRef = 64;    // reference MAX_VERTS: more vertices => status vertex_overflow
constexpr int kCapFast = 64;        // vertex / plane slots of a cell in shared memory
constexpr int kStackFast = 256;     // pending BVH nodes of a cell in shared memory
constexpr int kCapMid = 128;        // vertex / plane slots of a deferred cell (shared memory, second launch)
constexpr int kStackMid = 512;
constexpr int kCapBig = 256;        // vertex / plane slots of a cell that outgrew kCapMid (global memory)
constexpr int kStackBig = 1024;     // traversal stack of a deferred cell
constexpr int kCapHuge = 512;       // vertex / plane slots of a cell that outgrew kCapBig (rare)
constexpr int kStackHuge = 2048;
constexpr int kHugeSlabs = 256;     // such cells per build (global-memory state each)
constexpr int kRowWidth = 36;       // row slots per cell: a cell with <= 64 vertices has <= 34 faces
constexpr int kBigRowWidth = kCapBig; // row slots of a deferred cell
#ifndef PG_WARPS_PER_BLOCK
#define PG_WARPS_PER_BLOCK 8
#endif
constexpr int kWarpsPerBlock = PG_WARPS_PER_BLOCK; // cell kernel block, one cell per warp at a time
constexpr int kMaxWarpsPerSM = 32;  // upper bound of resident cell warps per SM (grid cap of the first pass)
constexpr int kBigWarps = 4;        // warps per block of the 256-slot tier (state in shared memory)
constexpr int kMidWarps = 4;        // warps per block of the 128-slot tier (13 KB of shared memory each)
constexpr int kMidBlocksPerSM = 3;  // its resident blocks per SM (up to 170 registers per thread)
constexpr int kMaxLeaf = 32;        // leaf size limit (one candidate per lane)
constexpr int kDefaultLeaf = 16;
constexpr int kWindow = 16;         // optional warm start: sorted neighbours i-16 .. i+16
constexpr uint32_t kBigFlag = 0x40000000u; // deg[] flag: row lives in the deferred-row area

// statistics counters (uint64 each) in the workspace
enum Stat : int
{
    kStatTests = 0,      // FP32 side tests
    kStatFp64 = 1,       // tests escalated past the FP32 filter
    kStatExpansion = 2,  // tests escalated past the FP64 filter
    kStatDeferred = 3,   // cells deferred to the large-capacity pass
    kStatNodes = 4,      // BVH nodes visited
    kStatLeaves = 5,     // leaves visited
    kStatClips = 6,      // clips that changed a cell
    kStatCandidates = 7, // candidates that reached the vertex test
    // SM cycles per phase, summed over warps (only with profiling enabled)
    kStatCycCell = 8,    // whole cell
    kStatCycWarm = 9,    // warm-start / initial-guess batches
    kStatCycNodes = 10,  // BVH node tests
    kStatCycLeaves = 11, // leaf batches (pre-check + clips)
    kStatCycClips = 12,  // clips
    kStatCycOut = 13,    // row output
    kStatDeferVerts = 14,  // deferrals / large-pass overflows: vertex or plane slots
    kStatDeferStack = 15,  // deferrals / large-pass overflows: traversal stack
    kStatVertex64 = 16,    // vertices rebuilt in FP64 (ill-conditioned in FP32)
    kStatHintHit = 17,     // cells certified within their search radius after the radius dropped a node
    kStatHintMiss = 18,    // cells whose search radius was too small (a second, unbounded pass ran)
    kStatCycBig = 19,      // SM cycles of the 256/512-slot rebuilds (only with profiling enabled)
    kNumStats = 20,
};

// leaf reference encoding in BVH records: bit 31 set, count-1 in bits 26..30,
// first sorted point index in bits 0..25 (N < 2^26).
__host__ __device__ __forceinline__ int leaf_ref(int first, int count)
{
    return (int)(0x80000000u | ((uint32_t)(count - 1) << 26) | (uint32_t)first);
}
__host__ __device__ __forceinline__ bool ref_is_leaf(int r) { return r < 0; }
__host__ __device__ __forceinline__ int leaf_first(int r) { return r & 0x3FFFFFF; }
__host__ __device__ __forceinline__ int leaf_count(int r) { return ((r >> 26) & 31) + 1; }

constexpr int64_t kMaxPoints = (int64_t)1 << 26;

// cloud of a point (original order) or of a sorted slot: clouds are contiguous in both
__host__ __device__ __forceinline__ int cloud_of(const int *off, int num_clouds, int i)
{
    int lo = 0, hi = num_clouds;
    while (hi - lo > 1)
    {
        int mid = (lo + hi) >> 1;
        if (off[mid] <= i)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// float <-> order-preserving int for atomic min / max
__device__ __forceinline__ int float_to_ordered(float f)
{
    int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float ordered_to_float(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF); }

// ---------------------------------------------------------------------------
// Workspace: one caller-provided device buffer, carved into 256-byte aligned
// segments. The layout depends only on (N, weighted).
// ---------------------------------------------------------------------------
struct Workspace
{
    // small header
    int *bounds;          // [8 per cloud]: ordered-int min xyz, max xyz, max w, unused
    float *box;           // [8 per cloud]: reference box lo xyz, hi xyz, max weight
    float *morton;        // [4 per cloud]: Morton origin xyz, extent
    int *cloud_off;       // [clouds + 1]: first point of each cloud (original order = sorted order by cloud)
    int *cloud_root;      // [clouds]: BVH root reference of each cloud
    int *counters;        // [16]: work counter, deferred count, error flag, edge total (2 ints), ...
    unsigned long long *stats; // [kNumStats]
    // LBVH
    unsigned long long *keys0, *keys1;
    uint32_t *vals0, *vals1;
    uint32_t *hist;       // [256 * sort blocks]
    uint32_t *scan_tmp;   // block sums of the generic scan
    float4 *pts;          // [N] sorted points (x, y, z, w)
    int *oid;             // [N] sorted slot -> original index
    int *rank;            // [N] original index -> sorted slot
    int *left, *right;    // [N] Karras children (>= 0 internal, < 0: ~leaf point)
    int *first, *last;    // [N] range of each internal node
    int *parent_int;      // [N] parent of internal nodes
    int *parent_leaf;     // [N] parent of leaf points
    int *flags;           // [N] refit arrival counters
    float4 *nbox;         // [2N] internal node box lo(xyz)+maxw, hi(xyz)+count
    float4 *records;      // [4N] traversal records of internal nodes
    int *rparent;         // [N] record node -> its entry in its parent's record (parent << 1 | side)
    int *pleaf;           // [N] sorted point -> the entry of the leaf holding it (parent << 1 | side)
    float *hint;          // [N] search radius per sorted slot (learned or given), <= 0: none
    // cells
    int *rows;            // [N * kRowWidth] directed rows by original index
    int *deg;             // [N] directed degree by original index (kBigFlag: deferred row)
    int *big_list;        // [N] sorted slots deferred to the large-capacity passes
    int *big_list2;       // [big_cap] sorted slots that outgrew the middle tier too
    int *big_slot2;       // [big_cap] their deferred-row slots
    int *big_rows;        // [big_cap * kBigRowWidth]
    void *huge_slabs;     // [kHugeSlabs] state of cells that outgrew the large capacity
    // CSR
    int *cnt;             // [N] kept directed entries per row
    int *miss;            // [N] reverse entries to add per row
    int *fill;            // [N] fill cursors
    unsigned long long *rmask; // [2N] per directed row: entries kept, reverse entries to add
    uint32_t *sizes;      // [N+1] scan input / output
    size_t bytes;
};

int big_warps();   // upper bound of resident cell warps on the device
size_t huge_slab_bytes();
size_t workspace_layout(int64_t n, int num_clouds, char *base, Workspace *ws);

} // namespace pg
