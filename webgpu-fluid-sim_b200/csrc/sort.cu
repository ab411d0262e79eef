// sort.cu -- stable LSD radix sort of (Morton key, body id) pairs.
//
// Replaces the third-party webgpu-radix-sort@1.0.7 kernel that the reference
// dispatches at src/simulation.ts:400 (constructed at :132-140 with
// bit_count 32 over mortonCodes/bodyIndices).  The contract is the stable
// sort by key: equal keys keep ascending body id, which the index tie-break of
// the hierarchy build (lbvh.wgsl:78-80) then turns into a unique tree.
//
// Design (onesweep, one kernel per 8-bit digit):
//  - The digit histograms of every pass come from the encode kernel, so each
//    pass reads its keys exactly once.
//  - A CTA takes the next tile (kSortTile keys) from an atomic counter (so lower
//    tiles are always already running), ranks its keys warp by warp with a
//    ballot multisplit (stable: item-major, lane-minor = memory order),
//    publishes its per-digit counts, stages the tile in shared memory in
//    digit order, and then resolves its global offsets by a decoupled
//    look-back over the tiles before it, several tiles per round trip.  The
//    look-back spin is bounded; on giving up it raises kErrLookbackSpin
//    instead of hanging.
//  - Staged keys and ids are written out in runs, so global stores are
//    contiguous per digit.
//  - Pass 0 does not read ids: it writes the identity permutation of
//    lbvh.wgsl:68 directly.
//  - With an even number of passes (4 for 32-bit keys, 8 for 64-bit keys)
//    the result lands back in the public codes / ids buffers.
#include <cuda/atomic>

#include "bh_internal.cuh"

namespace bh {

constexpr uint32_t kFlagAggregate = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kFlagMask = 3u << 30;
constexpr uint32_t kValueMask = (1u << 30) - 1;
#ifndef BH_SORT_LOOK_BATCH
#define BH_SORT_LOOK_BATCH 4
#endif
constexpr int kLookBatch = BH_SORT_LOOK_BATCH;  // predecessor tiles read per look-back round

// Exclusive scan over the block (every thread takes part; threads past the
// 256 digits pass 0, so the digits' prefixes are unaffected by them).
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* s_tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_tot[warp] = x;
    __syncthreads();
    uint32_t before = 0;
#pragma unroll
    for (int w = 0; w < kRadix / 32; ++w)
        if (w < warp) before += s_tot[w];
    __syncthreads();
    return before + x - v;
}

#ifndef BH_SORT_MIN_BLOCKS
#define BH_SORT_MIN_BLOCKS 2
#endif

template <typename K, bool FIRST>
__global__ void __launch_bounds__(kSortThreads, BH_SORT_MIN_BLOCKS)
onesweep_kernel(const K* __restrict__ keys_in, const uint32_t* __restrict__ ids_in,
                K* __restrict__ keys_out, uint32_t* __restrict__ ids_out, uint32_t n, int pass,
                StepScratch* __restrict__ scratch, uint32_t* __restrict__ status, uint32_t tiles,
                uint32_t* __restrict__ err, uint32_t spin_cap, uint32_t debug_flags) {
    constexpr int W = kSortThreads / 32;
    __shared__ uint32_t s_whist[W][kRadix];
    __shared__ uint32_t s_tile_excl[kRadix];
    __shared__ uint32_t s_gbase[kRadix];
    __shared__ uint32_t s_tot[W];
    __shared__ uint32_t s_tile;
    extern __shared__ __align__(16) unsigned char s_dyn[];
    K* s_keys = reinterpret_cast<K*>(s_dyn);
    uint32_t* s_ids = reinterpret_cast<uint32_t*>(s_keys + kSortTile);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(&scratch->tile_ctr[pass], 1u);
    for (int i = lane; i < kRadix; i += 32) s_whist[warp][i] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t seg = tile * kSortTile + (uint32_t)warp * 32u * kSortItems;
    const int shift = pass * kRadixBits;

    K key[kSortItems];
    uint32_t id[kSortItems];
    uint32_t rank[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        uint32_t idx = seg + (uint32_t)k * 32u + (uint32_t)lane;
        if (idx < n) {
            key[k] = keys_in[idx];
            id[k] = FIRST ? idx : ids_in[idx];
        } else {
            key[k] = 0;
            id[k] = 0;
        }
    }
    // Warp-local stable ranking.  The lanes holding the same digit are found
    // by eight ballots, one per digit bit (warp multisplit): a constant cost,
    // where a match instruction slows down with the number of distinct
    // digits in the warp.
    const bool full_tile = tile * (uint32_t)kSortTile + (uint32_t)kSortTile <= n;
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        uint32_t idx = seg + (uint32_t)k * 32u + (uint32_t)lane;
        bool valid = idx < n;
        uint32_t d = (uint32_t)(key[k] >> shift) & 0xFFu;
        unsigned peers = full_tile ? 0xFFFFFFFFu : __ballot_sync(0xFFFFFFFFu, valid);
#pragma unroll
        for (int bit = 0; bit < kRadixBits; ++bit) {
            const bool on = (d >> bit) & 1u;
            const unsigned vote = __ballot_sync(0xFFFFFFFFu, on);
            peers &= on ? vote : ~vote;
        }
        if (!valid) peers = 1u << lane;
        int leader = __ffs(peers) - 1;
        uint32_t below = __popc(peers & ((1u << lane) - 1u));
        uint32_t base = 0;
        if (valid && lane == leader) {
            base = s_whist[warp][d];
            s_whist[warp][d] = base + (uint32_t)__popc(peers);
        }
        base = __shfl_sync(0xFFFFFFFFu, base, leader);
        rank[k] = base + below;
        __syncwarp();
    }
    __syncthreads();
    // Per digit (threads 0..255): exclusive prefix over warps, and the tile's count.
    static_assert(kSortThreads >= kRadix && kSortThreads % 32 == 0, "one thread per digit");
    const bool digit_thread = tid < kRadix;
    const uint32_t d = digit_thread ? (uint32_t)tid : 0u;
    uint32_t run = 0;
    if (digit_thread) {
#pragma unroll
        for (int w = 0; w < W; ++w) {
            uint32_t c = s_whist[w][d];
            s_whist[w][d] = run;
            run += c;
        }
    }
    const uint32_t tile_cnt = run;
    // Publish this tile's aggregate (or inclusive prefix for tile 0).
    uint32_t* my_status = status + ((size_t)pass * tiles + tile) * kRadix;
    if (digit_thread) {
        cuda::atomic_ref<uint32_t, cuda::thread_scope_device> a(my_status[d]);
        a.store((tile == 0 ? kFlagPrefix : kFlagAggregate) | tile_cnt, cuda::memory_order_relaxed);
    }
    const uint32_t tile_excl = block_excl_scan(tile_cnt, s_tot);
    const uint32_t glob_excl = block_excl_scan(digit_thread ? scratch->hist[pass][d] : 0u, s_tot);
    if (digit_thread) s_tile_excl[d] = tile_excl;
    __syncthreads();
    // Stage in digit order before the look-back: the tile's own work is done
    // while the tiles before it finish theirs, so the walk back is shorter.
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        uint32_t idx = seg + (uint32_t)k * 32u + (uint32_t)lane;
        if (idx < n) {
            uint32_t dd = (uint32_t)(key[k] >> shift) & 0xFFu;
            uint32_t p = s_tile_excl[dd] + s_whist[warp][dd] + rank[k];
            s_keys[p] = key[k];
            s_ids[p] = id[k];
        }
    }
    // Decoupled look-back over earlier tiles, one digit per thread, reading
    // kLookBatch tiles per round trip (nearest first): the values are used up
    // to the first inclusive prefix, and re-read from the first tile that has
    // not published yet.
    uint32_t excl = 0;
    if (tile > 0 && digit_thread) {
        uint32_t* st = status + (size_t)pass * tiles * kRadix + d;
        int t = (int)tile - 1;
        uint32_t spins = 0;
        while (true) {
            uint32_t v[kLookBatch];
#pragma unroll
            for (int j = 0; j < kLookBatch; ++j) {
                v[j] = kFlagPrefix;  // below tile 0: never used
                if (t - j >= 0) {
                    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> a(st[(size_t)(t - j) * kRadix]);
                    v[j] = a.load(cuda::memory_order_relaxed);
                }
            }
            // Test hook: tile 1 of the first pass never sees its only
            // predecessor, tile 0 (entry j = 0), publish.
            if (FIRST && (debug_flags & kDebugLookbackUnpublished) && tile == 1u) v[0] = 0u;
            bool done = false;
            int used = 0;
#pragma unroll
            for (int j = 0; j < kLookBatch; ++j) {
                if (done || used < j || (v[j] & kFlagMask) == 0u) continue;
                excl += v[j] & kValueMask;
                used = j + 1;
                done = (v[j] & kFlagMask) == kFlagPrefix || t - j == 0;
            }
            if (done) break;
            t -= used;
            if (used == 0) {
                if (++spins > spin_cap) {
                    atomicOr(err, kErrLookbackSpin);
                    break;
                }
                if (spins > 64) __nanosleep(64);
            }
        }
        cuda::atomic_ref<uint32_t, cuda::thread_scope_device> a(my_status[d]);
        a.store(kFlagPrefix | (excl + tile_cnt), cuda::memory_order_relaxed);
    }
    if (digit_thread) s_gbase[d] = glob_excl + excl;
    __syncthreads();
    const uint32_t tile_base = tile * kSortTile;
    const uint32_t tile_n = (n - tile_base) < (uint32_t)kSortTile ? (n - tile_base) : (uint32_t)kSortTile;
    for (uint32_t i = (uint32_t)tid; i < tile_n; i += kSortThreads) {
        K kk = s_keys[i];
        uint32_t dd = (uint32_t)(kk >> shift) & 0xFFu;
        uint32_t dst = s_gbase[dd] + (i - s_tile_excl[dd]);
        // Offsets are in range unless a look-back gave up; never write outside.
        if (dst < n) {
            keys_out[dst] = kk;
            ids_out[dst] = s_ids[i];
        } else {
            atomicOr(err, kErrLookbackSpin);
        }
    }
}

// One pass per key byte, or fewer (an even count) when the high bytes are
// known to be zero (ensemble keys: system id above a 32-bit Morton code).
int sort_passes(const DeviceBuffers& b) { return b.sort_passes > 0 ? b.sort_passes : b.key_bytes; }

template <typename K>
static void sort_impl(const DeviceBuffers& b, cudaStream_t s) {
    const size_t smem = (size_t)kSortTile * (sizeof(K) + sizeof(uint32_t));
    const int passes = sort_passes(b);
    K* kin = (K*)b.codes;
    K* kout = (K*)b.codes_alt;
    uint32_t* iin = b.ids;
    uint32_t* iout = b.ids_alt;
    for (int p = 0; p < passes; ++p) {
        if (p == 0)
            onesweep_kernel<K, true><<<b.tiles, kSortThreads, smem, s>>>(
                kin, nullptr, kout, iout, b.n, p, b.scratch, b.status, b.tiles, b.err, b.spin_cap,
                b.debug_flags);
        else
            onesweep_kernel<K, false><<<b.tiles, kSortThreads, smem, s>>>(
                kin, iin, kout, iout, b.n, p, b.scratch, b.status, b.tiles, b.err, b.spin_cap,
                b.debug_flags);
        K* tk = kin; kin = kout; kout = tk;
        uint32_t* ti = iin; iin = iout; iout = ti;
    }
}

template <typename K>
static cudaError_t set_sort_attributes() {
    const int smem = (int)((size_t)kSortTile * (sizeof(K) + sizeof(uint32_t)));
    cudaError_t e = cudaFuncSetAttribute(onesweep_kernel<K, true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(onesweep_kernel<K, false>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

// Opt the sort kernels into more than 48 KB of dynamic shared memory on the
// current device (called once per device before any launch or capture).
cudaError_t sort_init_attributes() {
    cudaError_t e = set_sort_attributes<uint32_t>();
    if (e != cudaSuccess) return e;
    return set_sort_attributes<uint64_t>();
}

void launch_sort(const DeviceBuffers& b, cudaStream_t s) {
    if (b.n == 0) return;
    if (b.key_bytes == 8) sort_impl<uint64_t>(b, s);
    else sort_impl<uint32_t>(b, s);
}

}  // namespace bh
