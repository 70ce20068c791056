// String hashing without any device allocation.
//
// Some callers cannot allocate device memory: a library embedded in a host process that
// owns all device memory through its own pool (a database or query-engine plugin, for
// example), or a latency-critical serving thread that must not call cudaMalloc because it
// can synchronise the device and stall unrelated streams. rsb_hash_strings_static gives
// them the device string hash of rsb_hash_strings: it stages the keys, hashes them with the
// same kernel and copies the hashes back, all inside one fixed array of device memory that
// is part of this library's image.
//
// The array is a file-scope __device__ variable, so every GPU that loads the library holds
// it (kStaticScratchBytes, about 1.8 MiB) until the process exits. It comes into existence
// when the CUDA runtime loads this library's device code on a device: at the first call
// under lazy module loading (the CUDA 12 default), or when the context is created under
// CUDA_MODULE_LOADING=EAGER. A caller whose memory pool will claim all device memory should
// therefore make one small call on each device before the pool takes the memory. All calls
// on a device share the array and it keeps the last call's contents. The kernel reads only
// bytes the same call has just copied in and every hash it writes is copied out, so nothing
// needs clearing between calls. Two calls whose GPU work overlapped would race on the array;
// this entry point prevents that by holding a process-wide lock until its stream has
// finished. The first call on a device resolves the array's device address with
// cudaGetSymbolAddress (with that device current); make that first call before any stream
// capture begins. Every call copies through pageable host memory and waits for its stream,
// so a call whose stream is capturing is refused (RSB_ERR_BAD_ARG) before any work, which
// leaves the caller's capture intact. Limits: 32,768 keys and 1 MiB of key bytes per call,
// counted from offsets[0] (key i is bytes[offsets[i] .. offsets[i+1]), and only
// bytes[offsets[0] .. offsets[n]) is copied).
#include <cstring>
#include <mutex>

#include "rsb_kernels.cuh"

namespace rsb {
namespace {

constexpr uint64_t kStaticMaxKeys = 1ull << 15;   // keys per call
constexpr uint64_t kStaticMaxBytes = 1ull << 20;  // key bytes per call
constexpr size_t kOffBytes = 0;
constexpr size_t kOffOffsets = kStaticMaxBytes;                            // 8-byte aligned
constexpr size_t kOffHashes = kOffOffsets + (kStaticMaxKeys + 1) * 8 + 8;  // 16-byte aligned
constexpr size_t kStaticScratchBytes = kOffHashes + kStaticMaxKeys * 16;
static_assert(kOffHashes % 16 == 0, "hash output must be 16-byte aligned");

static __device__ __align__(256) uint8_t g_static_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
uint8_t *g_static_ptr[kMaxDevices] = {};

// Resolves the device address of g_static_scratch on the current device (once per device).
// The host-side symbol is only a stand-in; kernels must receive this address.
cudaError_t static_scratch(int dev, uint8_t **out) {
    if (!g_static_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return e;
        g_static_ptr[dev] = (uint8_t *)p;
    }
    *out = g_static_ptr[dev];
    return cudaSuccess;
}

}  // namespace
}  // namespace rsb

extern "C" rsb_status rsb_hash_strings_static(const uint8_t *bytes, const uint64_t *offsets, uint64_t n,
                                              rsb_hash128 *out, void *stream) {
    using namespace rsb;
    if (!offsets || (n && !out)) return RSB_ERR_BAD_ARG;
    if (n > kStaticMaxKeys) return RSB_ERR_BAD_ARG;  // more keys than the static array holds
    for (uint64_t i = 0; i < n; ++i)
        if (offsets[i + 1] < offsets[i]) return RSB_ERR_BAD_ARG;
    const uint64_t first = offsets[0];
    const uint64_t nbytes = offsets[n] - first;  // offsets are non-decreasing (checked above)
    if (nbytes > kStaticMaxBytes) return RSB_ERR_BAD_ARG;
    if (nbytes && !bytes) return RSB_ERR_BAD_ARG;
    if (n == 0) return RSB_OK;
    // An error left pending on this thread by earlier, unrelated CUDA work is not ours to
    // report or clear: refuse the call and leave it in place for its owner.
    if (cudaPeekAtLastError() != cudaSuccess) return RSB_ERR_CUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return RSB_ERR_NO_DEVICE;
    }
    cudaStream_t st = (cudaStream_t)stream;
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &capture) != cudaSuccess) {
        cudaGetLastError();
        return RSB_ERR_CUDA;
    }
    if (capture != cudaStreamCaptureStatusNone) return RSB_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lock(g_static_mu);
    uint8_t *base = nullptr;
    if (static_scratch(dev, &base) != cudaSuccess) {
        cudaGetLastError();
        return RSB_ERR_CUDA;
    }
    uint8_t *d_bytes = base + kOffBytes;
    uint64_t *d_offsets = (uint64_t *)(base + kOffOffsets);
    uint64_t *d_hashes = (uint64_t *)(base + kOffHashes);
    bool ok = true;
    if (nbytes) ok &= cudaMemcpyAsync(d_bytes, bytes + first, nbytes, cudaMemcpyHostToDevice, st) == cudaSuccess;
    ok &= cudaMemcpyAsync(d_offsets, offsets, (n + 1) * 8, cudaMemcpyHostToDevice, st) == cudaSuccess;
    if (ok) {
        // the kernel reads key i at d_bytes[offsets[i] - first]
        launch_hash_strings(d_bytes, d_offsets, n, first, d_hashes, st);
        ok &= cudaGetLastError() == cudaSuccess;  // nothing was pending at entry: this launch's own status
    }
    if (ok) ok &= cudaMemcpyAsync(out, d_hashes, n * 16, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok &= cudaStreamSynchronize(st) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        return RSB_ERR_CUDA;
    }
    return RSB_OK;
}
