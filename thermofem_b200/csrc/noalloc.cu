// noalloc.cu -- exclusive prefix sum that allocates nothing.
//
// tf_scan_exclusive_i32 takes its per-tile partial sums from stream-ordered
// temporary allocations.  Some callers cannot allocate device memory at the
// time they need a scan: code running inside another library's allocator or
// memory-pool callback, code holding a fixed device-memory budget that must
// not grow, or hosts where cudaMalloc may block on a device-wide
// synchronisation they cannot afford.  tf_scan_exclusive_i32_noalloc gives
// them the same result with its scratch in a fixed array compiled into this
// library: every device that loads the library reserves it (256 KB) until
// the process exits.
//
// Limits and sharing: n may be at most kMaxItems (2^27 = 134,217,728).  All
// calls on a device share the one array, and it keeps whatever the last call
// left in it; each call writes every scratch word before reading it, so no
// clearing is needed between calls, but two calls whose kernels overlap on
// the GPU (different streams, no ordering between them) race on the array and
// both results are undefined.
//
// First call on a device: CUDA loads a library's kernels lazily (the default
// since CUDA 12.2), so the first call on each device loads this module, which
// allocates the array and the module's code on the device and may
// synchronise it, and then looks up the array's device address.  A caller
// that must not allocate at all makes that first call beforehand, at a point
// where allocating is allowed (and outside any stream capture); every later
// call on that device allocates nothing.  The address is kept per device
// ordinal for the life of the process: after cudaDeviceReset the device's
// memory, the array included, is gone, so the function must not be called
// again in that process.
#include <mutex>

#include "common.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int64_t kTile = kThreads * kItems;            // 2048 items per tile
constexpr int64_t kMaxTiles = 65536;                    // first-level tile sums
constexpr int64_t kMaxItems = kTile * kMaxTiles;        // 2^27
constexpr int64_t kMaxTiles2 = (kMaxTiles + kTile - 1) / kTile;  // 32 second-level sums

// Scratch: first-level tile sums, then second-level tile sums.
static __device__ __align__(256) int32_t g_scan_scratch[kMaxTiles + kMaxTiles2];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
int32_t *g_scratch_address[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device (the host-side name of the array is not a device address).
int32_t *scratch_address(int device) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_address[device]) {
        void *p = nullptr;
        tfb::cuda_check(cudaGetSymbolAddress(&p, g_scan_scratch), "cudaGetSymbolAddress(scan scratch)");
        g_scratch_address[device] = static_cast<int32_t *>(p);
    }
    return g_scratch_address[device];
}

__device__ __forceinline__ void tile_scan(int (&v)[kItems]) {
    __shared__ int warp_total[kThreads / 32];
    int local = 0;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const int t = v[k];
        v[k] = local;
        local += t;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inc = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) warp_total[warp] = inc;
    __syncthreads();
    int before = 0;
    for (int w = 0; w < warp; ++w) before += warp_total[w];
    const int prefix = before + inc - local;
#pragma unroll
    for (int k = 0; k < kItems; ++k) v[k] += prefix;
}

// Sum of each tile of `in` into sums[tile].
__global__ void __launch_bounds__(kThreads) tile_sums(int64_t n, const int32_t *__restrict__ in,
                                                       int32_t *__restrict__ sums) {
    __shared__ int warp_total[kThreads / 32];
    const int64_t base = blockIdx.x * kTile + static_cast<int64_t>(threadIdx.x) * kItems;
    int s = 0;
#pragma unroll
    for (int k = 0; k < kItems; ++k)
        if (base + k < n) s += in[base + k];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) warp_total[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kThreads / 32; ++w) t += warp_total[w];
        sums[blockIdx.x] = t;
    }
}

// Exclusive scan of each tile plus the tile's offset (offsets null: 0).
__global__ void __launch_bounds__(kThreads) tile_scan_add(int64_t n, const int32_t *in, int32_t *out,
                                                           const int32_t *__restrict__ offsets) {
    const int64_t base = blockIdx.x * kTile + static_cast<int64_t>(threadIdx.x) * kItems;
    int v[kItems];
#pragma unroll
    for (int k = 0; k < kItems; ++k) v[k] = base + k < n ? in[base + k] : 0;
    tile_scan(v);
    const int add = offsets ? offsets[blockIdx.x] : 0;
#pragma unroll
    for (int k = 0; k < kItems; ++k)
        if (base + k < n) out[base + k] = v[k] + add;
}

}  // namespace

extern "C" int tf_scan_exclusive_i32_noalloc(void *stream, int64_t n, const int32_t *in, int32_t *out) {
    return tfb::guard([&] {
        tfb::require(n >= 0, "negative size");
        if (n > kMaxItems)
            tfb::fail(TF_ERR_LENGTH, "tf_scan_exclusive_i32_noalloc: n exceeds the fixed scratch limit of 134217728 items");
        if (n == 0) return;
        tfb::require(in != nullptr && out != nullptr, "null array");
        int device = 0;
        tfb::cuda_check(cudaGetDevice(&device), "cudaGetDevice");
        tfb::require(device >= 0 && device < kMaxDevices, "device ordinal beyond the scratch table");
        int32_t *sums = scratch_address(device);
        int32_t *sums2 = sums + kMaxTiles;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const int64_t tiles = (n + kTile - 1) / kTile;
        if (tiles == 1) {
            tile_scan_add<<<1, kThreads, 0, s>>>(n, in, out, nullptr);
        } else {
            tile_sums<<<static_cast<unsigned>(tiles), kThreads, 0, s>>>(n, in, sums);
            const int64_t tiles2 = (tiles + kTile - 1) / kTile;
            if (tiles2 == 1) {
                tile_scan_add<<<1, kThreads, 0, s>>>(tiles, sums, sums, nullptr);
            } else {
                tile_sums<<<static_cast<unsigned>(tiles2), kThreads, 0, s>>>(tiles, sums, sums2);
                tile_scan_add<<<1, kThreads, 0, s>>>(tiles2, sums2, sums2, nullptr);
                tile_scan_add<<<static_cast<unsigned>(tiles2), kThreads, 0, s>>>(tiles, sums, sums, sums2);
            }
            tile_scan_add<<<static_cast<unsigned>(tiles), kThreads, 0, s>>>(n, in, out, sums);
        }
        tfb::cuda_check(cudaGetLastError(), "tf_scan_exclusive_i32_noalloc launch");
    });
}
