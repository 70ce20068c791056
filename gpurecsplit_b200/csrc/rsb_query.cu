// Device evaluation of operator() for many keys (bijection checks of large builds).
#include "rsb_kernels.cuh"
#include "rsb_query.cuh"

namespace rsb {

namespace {
__global__ void k_query(MphfView f, const ulonglong2 *__restrict__ keys, uint64_t n, uint64_t *__restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const ulonglong2 k = keys[i];
        out[i] = mphf_query(f, k.x, k.y);
    }
}
}  // namespace

void launch_query_view(const MphfView &f, const uint64_t *keys128, uint64_t n, uint64_t *out, cudaStream_t st) {
    uint64_t g = (n + 255) / 256;
    if (g < 1) g = 1;
    if (g > device_sm_count() * 16) g = device_sm_count() * 16;
    use_max_smem(k_query);
    k_query<<<(int)g, 256, 0, st>>>(f, (const ulonglong2 *)keys128, n, out);
}

}  // namespace rsb
