// k_sort.cu — stable LSD radix sort of (key, id) pairs for the hash grid.
//
// Replaces the reference's CS_RadixHistogram / CS_RadixPrefixSum /
// CS_RadixScatter chain (src/fluid/PBFluids.cpp:354-405), which sorts all 32
// key bits in four 8-bit passes with a single-workgroup serial scan.  Here:
//   * only ceil(log2(H)) bits are sorted (keys are masked to H-1, so higher
//     digits are zero and those passes are identities — the permutation is
//     bit-identical);
//   * each pass is upsweep (per-tile digit counts in shared memory) ->
//     device-wide scan (one block per digit) -> downsweep (warp match-any
//     ranking, tile reordered in shared memory, coalesced scatter);
//   * ranks are stable: within a tile by (warp, round, lane) = input order,
//     across tiles by the digit-major / tile-minor scan, exactly the order the
//     reference's column-major histogram + ballot ranking produces.
#include "pbf_kernels.h"

namespace pbf {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 keys per tile
static_assert(kSortTile == (int)kSortTileKeys, "scratch sizing elsewhere uses kSortTileKeys");
constexpr int kRadix = 256;
constexpr int kWarps = kSortThreads / 32;

uint32_t sort_num_tiles(uint32_t n) { return (n + kSortTile - 1) / kSortTile; }

__global__ void __launch_bounds__(kSortThreads) k_sort_upsweep(const uint32_t* __restrict__ keys, uint32_t n,
                                                              int shift, uint32_t dmask, uint32_t* __restrict__ hist,
                                                              uint32_t num_tiles)
{
    __shared__ uint32_t cnt[kWarps][kRadix];
    const int warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kWarps * kRadix; i += kSortThreads) (&cnt[0][0])[i] = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * kSortTile;
    // all of the thread's loads are issued before its first shared-memory
    // atomic, so they are in flight together
    uint32_t k[kSortItems];
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint32_t idx = base + r * kSortThreads + threadIdx.x;
        k[r] = idx < n ? __ldg(keys + idx) : 0xffffffffu;
    }
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint32_t idx = base + r * kSortThreads + threadIdx.x;
        if (idx < n) atomicAdd(&cnt[warp][(k[r] >> shift) & dmask], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += kSortThreads) {
        uint32_t s = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) s += cnt[w][d];
        hist[(size_t)d * num_tiles + blockIdx.x] = s;
    }
}

// Exclusive scan of one digit's per-tile counts (block = digit); writes the
// digit total.
__global__ void __launch_bounds__(1024) k_sort_scan(uint32_t* __restrict__ hist, uint32_t num_tiles,
                                                    uint32_t* __restrict__ totals)
{
    __shared__ uint32_t warp_sums[32];
    uint32_t* h = hist + (size_t)blockIdx.x * num_tiles;
    const uint32_t chunk = (num_tiles + 1023u) / 1024u;
    const uint32_t begin = threadIdx.x * chunk;
    const uint32_t end = min(begin + chunk, num_tiles);
    uint32_t local = 0;
    for (uint32_t i = begin; i < end; ++i) local += h[i];
    // block exclusive scan of `local`
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_sums[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        warp_sums[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    uint32_t run = incl - local + (warp ? warp_sums[warp - 1] : 0u);
    for (uint32_t i = begin; i < end; ++i) {
        const uint32_t v = h[i];
        h[i] = run;
        run += v;
    }
    if (threadIdx.x == 1023) totals[blockIdx.x] = warp_sums[31];
}

// Block-wide exclusive scan of one value per thread (256 threads).
__device__ __forceinline__ uint32_t block_exclusive_scan_256(uint32_t v, uint32_t* smem_warp /*[8]*/,
                                                             uint32_t* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) smem_warp[warp] = incl;
    __syncthreads();
    uint32_t off = 0, all = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        const uint32_t s = smem_warp[w];
        if (w < warp) off += s;
        all += s;
    }
    __syncthreads();
    if (total) *total = all;
    return off + incl - v;
}

__global__ void __launch_bounds__(kSortThreads) k_sort_downsweep(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ ids_in, uint32_t* __restrict__ keys_out,
    uint32_t* __restrict__ ids_out, uint32_t n, int shift, uint32_t dmask, const uint32_t* __restrict__ hist,
    const uint32_t* __restrict__ totals, uint32_t num_tiles)
{
    __shared__ uint32_t s_gbase[kRadix];       // global destination of this tile's first item of digit d
    __shared__ uint32_t s_wcnt[kWarps][kRadix];  // per-warp digit counts -> per-warp digit offsets
    __shared__ uint32_t s_bstart[kRadix];      // digit start inside the tile
    __shared__ uint32_t s_warp[kWarps];
    __shared__ uint32_t s_keys[kSortTile];
    __shared__ uint32_t s_ids[kSortTile];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile = blockIdx.x;
    const uint32_t base = tile * kSortTile;

    // digit bases: exclusive scan of the digit totals + this tile's prefix
    {
        const int d = threadIdx.x;  // kSortThreads == kRadix
        const uint32_t ex = block_exclusive_scan_256(__ldg(totals + d), s_warp, nullptr);
        s_gbase[d] = ex + __ldg(hist + (size_t)d * num_tiles + tile);
    }
    for (int i = threadIdx.x; i < kWarps * kRadix; i += kSortThreads) (&s_wcnt[0][0])[i] = 0;
    __syncthreads();

    // load: warp w owns items [w*32*kSortItems, (w+1)*32*kSortItems) of the tile, round-major
    uint32_t key[kSortItems], id[kSortItems], rank[kSortItems];
    const uint32_t wbase = base + warp * (32 * kSortItems);
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint32_t idx = wbase + r * 32 + lane;
        if (idx < n) {
            key[r] = __ldg(keys_in + idx);
            id[r] = ids_in ? __ldg(ids_in + idx) : idx;
        } else {
            key[r] = 0xffffffffu;
            id[r] = 0;
        }
    }
    // stable warp-level ranking with match-any
    const uint32_t lt_mask = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint32_t idx = wbase + r * 32 + lane;
        const bool valid = idx < n;
        const uint32_t d = valid ? ((key[r] >> shift) & dmask) : 0xffffffffu;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        uint32_t before = 0;
        if (valid) before = s_wcnt[warp][d];
        __syncwarp();
        if (valid && (peers & lt_mask) == 0) s_wcnt[warp][d] = before + __popc(peers);
        __syncwarp();
        rank[r] = before + __popc(peers & lt_mask);
    }
    __syncthreads();
    // per-digit: exclusive offsets across warps, and the tile's digit counts
    {
        const int d = threadIdx.x;
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t c = s_wcnt[w][d];
            s_wcnt[w][d] = run;
            run += c;
        }
        const uint32_t st = block_exclusive_scan_256(run, s_warp, nullptr);
        s_bstart[d] = st;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint32_t idx = wbase + r * 32 + lane;
        if (idx < n) {
            const uint32_t d = (key[r] >> shift) & dmask;
            const uint32_t lp = s_bstart[d] + s_wcnt[warp][d] + rank[r];
            s_keys[lp] = key[r];
            s_ids[lp] = id[r];
        }
    }
    __syncthreads();
    const uint32_t count = min((uint32_t)kSortTile, n - base);
    for (uint32_t i = threadIdx.x; i < count; i += kSortThreads) {
        const uint32_t k = s_keys[i];
        const uint32_t d = (k >> shift) & dmask;
        const uint32_t dst = s_gbase[d] + (i - s_bstart[d]);
        keys_out[dst] = k;
        ids_out[dst] = s_ids[i];
    }
}

// Same sort, with the result guaranteed to land in (out_k, out_i): the first
// pass writes to whichever pair makes the last pass end there, so the
// caller's output arrays double as one half of the ping-pong and only one
// more pair of scratch arrays is needed.
void launch_radix_sort_into(uint32_t n, uint32_t key_bits, const uint32_t* keys_in, uint32_t* out_k, uint32_t* out_i,
                            uint32_t* tmp_k, uint32_t* tmp_i, uint32_t* hist, uint32_t* totals, cudaStream_t st)
{
    if (key_bits == 0) key_bits = 1;
    const uint32_t passes = (key_bits + 7u) / 8u;
    const bool odd = (passes & 1u) != 0;
    uint32_t *rk = nullptr, *ri = nullptr;
    launch_radix_sort(n, key_bits, keys_in, odd ? out_k : tmp_k, odd ? out_i : tmp_i, odd ? tmp_k : out_k,
                      odd ? tmp_i : out_i, hist, totals, &rk, &ri, st, nullptr);
}

// Sorts keys_in (particle order, left untouched) with ids 0..n-1, ping-ponging
// between the (ka, ia) and (kb, ib) buffers; *out_keys / *out_ids receive the
// pair holding the result.
void launch_radix_sort(uint32_t n, uint32_t key_bits, const uint32_t* keys_in, uint32_t* ka, uint32_t* ia,
                       uint32_t* kb, uint32_t* ib, uint32_t* hist, uint32_t* totals, uint32_t** out_keys,
                       uint32_t** out_ids, cudaStream_t st, uint64_t* launches)
{
    const uint32_t num_tiles = sort_num_tiles(n);
    if (key_bits == 0) key_bits = 1;
    const uint32_t passes = (key_bits + 7u) / 8u;
    const uint32_t* kin = keys_in;
    const uint32_t* iin = nullptr;  // identity ids on the first pass
    uint32_t* kout = ka;
    uint32_t* iout = ia;
    int shift = 0;
    for (uint32_t p = 0; p < passes; ++p) {
        const uint32_t bits = (key_bits - (uint32_t)shift + (passes - p) - 1u) / (passes - p);
        const uint32_t dmask = (1u << bits) - 1u;
        k_sort_upsweep<<<num_tiles, kSortThreads, 0, st>>>(kin, n, shift, dmask, hist, num_tiles);
        k_sort_scan<<<kRadix, 1024, 0, st>>>(hist, num_tiles, totals);
        k_sort_downsweep<<<num_tiles, kSortThreads, 0, st>>>(kin, iin, kout, iout, n, shift, dmask, hist, totals,
                                                             num_tiles);
        if (launches) *launches += 3;
        shift += (int)bits;
        kin = kout;
        iin = iout;
        kout = (kout == ka) ? kb : ka;
        iout = (iout == ia) ? ib : ia;
    }
    *out_keys = const_cast<uint32_t*>(kin);
    *out_ids = const_cast<uint32_t*>(iin);
}

}  // namespace pbf
