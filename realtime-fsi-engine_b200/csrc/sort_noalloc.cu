// sort_noalloc.cu — the hash-key radix sort for callers that cannot allocate.
//
// Some callers of this library cannot call cudaMalloc: code that runs inside
// another framework's allocator (memory pools that own the whole device),
// plugins that are only handed device buffers, and real-time loops that must
// not enter the driver's allocator once running.  For them,
// pbf_sort_keys_noalloc sorts caller-provided device buffers and takes its
// scratch space (one ping-pong pair of key/id arrays plus the per-tile digit
// histograms) from a fixed array in this file instead of allocating it.
//
// Limits and sharing:
//   * at most PBF_NOALLOC_MAX_KEYS keys per call (about 8.3 MB of scratch,
//     held by every GPU that loads this library until the process exits);
//   * every call uses the same array; nothing in it has to start at zero
//     (each pass rewrites the histograms and totals it reads), but two calls
//     whose GPU work overlaps — on different streams, or from different host
//     threads — race on the array and corrupt each other's results;
//   * the stream must belong to the current device (the scratch address is
//     the current device's); a stream of another device is rejected.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/pbf_b200.h"
#include "pbf_engine.h"
#include "pbf_kernels.h"

namespace {

constexpr uint32_t kTile = pbf::kSortTileKeys;  // keys per sort tile (k_sort.cu)
constexpr uint32_t kMaxTiles = (PBF_NOALLOC_MAX_KEYS + kTile - 1) / kTile;
// layout: tmp keys | tmp ids | histograms (256 per tile) | digit totals (256)
constexpr size_t kScratchWords = 2u * PBF_NOALLOC_MAX_KEYS + 256u * kMaxTiles + 256u;

// Device-side scratch.  In host code this name is only a stand-in for the
// symbol; its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) uint32_t g_sort_scratch[kScratchWords];

// True when the n-word arrays at a and b share any word.
bool overlaps(const void* a, const void* b, uint32_t n)
{
    const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
    const uintptr_t len = (uintptr_t)n * sizeof(uint32_t);
    return x < y + len && y < x + len;
}

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint32_t* g_ptr[kMaxDevices] = {};

// Resolves the device address of g_sort_scratch on the current device (once
// per device).  This is the only call that may load the library's module on
// that device, so the first call of the entry point on a device must not be
// made while a stream on that device is being captured into a CUDA graph.
int scratch_for_current_device(cudaStream_t st, uint32_t** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return pbf::set_error(PBF_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return pbf::set_error(PBF_ERR_INVALID, "device %d out of range", dev);
    if (st) {
        int sdev = -1;
        e = cudaStreamGetDevice(st, &sdev);
        if (e != cudaSuccess) return pbf::set_error(PBF_ERR_INVALID, "cudaStreamGetDevice: %s", cudaGetErrorString(e));
        if (sdev != dev)
            return pbf::set_error(PBF_ERR_INVALID,
                                  "pbf_sort_keys_noalloc: stream belongs to device %d, current device is %d", sdev, dev);
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess || !p)
            return pbf::set_error(PBF_ERR_CUDA, "cudaGetSymbolAddress(sort scratch): %s", cudaGetErrorString(e));
        g_ptr[dev] = static_cast<uint32_t*>(p);
    }
    *out = g_ptr[dev];
    return PBF_OK;
}

}  // namespace

extern "C" int pbf_sort_keys_noalloc(const uint32_t* keys_dev, uint32_t n, uint32_t key_bits, uint32_t* sorted_keys_dev,
                                     uint32_t* sorted_ids_dev, void* stream)
{
    if (n == 0) return PBF_OK;
    if (!keys_dev || !sorted_keys_dev || !sorted_ids_dev) return pbf::set_error(PBF_ERR_INVALID, "null device pointer");
    if (n > PBF_NOALLOC_MAX_KEYS)
        return pbf::set_error(PBF_ERR_INVALID, "pbf_sort_keys_noalloc: %u keys exceed the fixed scratch of %u keys", n,
                              (uint32_t)PBF_NOALLOC_MAX_KEYS);
    if (key_bits > 32) return pbf::set_error(PBF_ERR_INVALID, "key_bits %u > 32", key_bits);
    // An odd number of digit passes writes the first pass straight into the
    // outputs while other tiles still read the keys, and the key and id
    // outputs are written by the same passes: no two of the three may overlap.
    if (overlaps(keys_dev, sorted_keys_dev, n) || overlaps(keys_dev, sorted_ids_dev, n) ||
        overlaps(sorted_keys_dev, sorted_ids_dev, n))
        return pbf::set_error(PBF_ERR_INVALID, "pbf_sort_keys_noalloc: keys, sorted keys and sorted ids must not overlap");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint32_t* s = nullptr;
    int rc = scratch_for_current_device(st, &s);
    if (rc) return rc;
    const uint32_t tiles = (n + kTile - 1) / kTile;
    uint32_t* tmp_k = s;
    uint32_t* tmp_i = s + PBF_NOALLOC_MAX_KEYS;
    uint32_t* hist = s + 2u * PBF_NOALLOC_MAX_KEYS;
    uint32_t* totals = hist + 256u * tiles;
    pbf::launch_radix_sort_into(n, key_bits, keys_dev, sorted_keys_dev, sorted_ids_dev, tmp_k, tmp_i, hist, totals, st);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return pbf::set_error(PBF_ERR_CUDA, "pbf_sort_keys_noalloc: %s", cudaGetErrorString(e));
    return PBF_OK;
}
