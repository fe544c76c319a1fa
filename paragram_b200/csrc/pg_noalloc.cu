// pg_noalloc.cu -- CSR offsets from per-row degrees without allocating device memory.
//
// Some callers cannot allocate device memory when they need this: deployments
// that fix their device-memory budget at start-up and forbid allocation calls
// afterwards, processes whose device memory is owned by another framework's
// allocator (so a foreign cudaMalloc is disallowed or fragments its pool), and
// latency-critical paths that cannot afford the implicit device
// synchronisation of cudaMalloc / cudaFree. For them this entry point runs the
// library's exclusive scan (pg_scan.cu) with its block-sum scratch in a
// file-scope device array instead of caller- or library-allocated memory.
//
// The array below is the whole scratch: kScratchWords 32-bit words (129 KB),
// enough for up to kMaxRows rows. Every GPU that loads the library holds one
// copy until the process exits. Every call on a device shares that copy and
// leaves the last call's block sums in it; nothing in it needs to start at
// zero, because each call writes every scratch word before reading it. Calls
// whose work overlaps on the GPU (different streams, or other host threads)
// race on the array and must be serialised by the caller.
#include <mutex>
#include <string>

#include "../../include/paragram_b200.h"
#include "pg_common.cuh"
#include "pg_kernels.cuh"

namespace pg
{

constexpr int64_t kMaxRows = ((int64_t)1 << 26) - 1; // same limit as the number of points
constexpr size_t kScratchWords = 33024;              // >= scan_tmp_elems(kMaxRows)

static __device__ __align__(256) uint32_t g_scan_scratch[kScratchWords];

// Host-side device address of g_scan_scratch, resolved once per device.
static std::mutex g_scratch_mutex;
static void *g_scratch_addr[256] = {nullptr};

static int scratch_address(uint32_t **out, std::string &err)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 256)
    {
        err = std::string("no usable current CUDA device: ") + cudaGetErrorString(e);
        return PG_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev])
    {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scan_scratch);
        if (e != cudaSuccess || !p)
        {
            err = std::string("cudaGetSymbolAddress of the static scan scratch failed: ") + cudaGetErrorString(e);
            return PG_ERR_CUDA;
        }
        g_scratch_addr[dev] = p;
    }
    *out = (uint32_t *)g_scratch_addr[dev];
    return PG_OK;
}

int set_last_error(int code, const std::string &msg); // pg_api.cu

} // namespace pg

extern "C" int pg_degrees_to_offsets_noalloc(int64_t num_rows, const int32_t *degrees, int32_t *offsets, void *stream)
{
    using namespace pg;
    if (num_rows < 0 || num_rows > kMaxRows)
        return set_last_error(PG_ERR_INVALID, "num_rows must be in [0, " + std::to_string(kMaxRows) +
                                                  "]: the static scan scratch holds no more rows");
    if (!offsets || (num_rows > 0 && !degrees))
        return set_last_error(PG_ERR_INVALID, "degrees and offsets must not be NULL");
    if (scan_tmp_elems(num_rows) > kScratchWords)
        return set_last_error(PG_ERR_INVALID, "num_rows exceeds the static scan scratch");
    cudaGetLastError();
    uint32_t *scratch = nullptr;
    std::string err;
    int rc = scratch_address(&scratch, err);
    if (rc != PG_OK)
        return set_last_error(rc, err);
    exclusive_scan((const uint32_t *)degrees, (uint32_t *)offsets, num_rows, scratch, (cudaStream_t)stream);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return set_last_error(PG_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
    return set_last_error(PG_OK, "");
}
