// Device evaluation of operator() for many keys (bijection checks of large builds).
#include <algorithm>

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
// Self-verification of a finished build (RSB_VERIFY). Every bucket's double Elias-Fano entry
// decodes to the offsets it was built from, as the reference checks in its debug builds
// (DoubleEF.hpp:351-364); and every key maps to a distinct value in [0, n): with n keys that
// is a bijection. A failure sets RSB_ERR_INTERNAL with the bucket or key index.
__global__ void k_verify_ef(MphfView f, const uint64_t *__restrict__ acc, const uint64_t *__restrict__ pos, uint64_t nb,
                            DevStatus *status) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nb; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t c0, c1, p0;
        ef_get(f, i, c0, c1, p0);
        if (c0 != acc[i] || c1 != acc[i + 1] || p0 != pos[i]) set_error(status, RSB_ERR_INTERNAL, i);
    }
}

__global__ void k_verify_bijection(MphfView f, const ulonglong2 *__restrict__ keys, uint64_t n, uint32_t *seen,
                                   DevStatus *status) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const ulonglong2 k = keys[i];
        const uint64_t v = mphf_query(f, k.x, k.y);
        if (v >= n) {
            set_error(status, RSB_ERR_INTERNAL, i);
            continue;
        }
        const uint32_t bit = 1u << (v % 32);
        if (atomicOr(&seen[v / 32], bit) & bit) set_error(status, RSB_ERR_INTERNAL, i);
    }
}

}  // namespace

void launch_verify(const MphfView &f, const uint64_t *keys128, uint64_t n, const uint64_t *acc, const uint64_t *pos,
                   uint64_t nb, uint32_t *seen, DevStatus *status, cudaStream_t st) {
    const int cap = device_sm_count() * 16;
    use_max_smem(k_verify_ef);
    k_verify_ef<<<(int)std::min<uint64_t>(cap, (nb + 255) / 256 + 1), 256, 0, st>>>(f, acc, pos, nb, status);
    cudaMemsetAsync(seen, 0, ((n + 31) / 32) * sizeof(uint32_t), st);
    use_max_smem(k_verify_bijection);
    k_verify_bijection<<<(int)std::min<uint64_t>(cap, (n + 255) / 256 + 1), 256, 0, st>>>(
        f, (const ulonglong2 *)keys128, n, seen, status);
    count_launches(2);
}

void launch_query_view(const MphfView &f, const uint64_t *keys128, uint64_t n, uint64_t *out, cudaStream_t st) {
    uint64_t g = (n + 255) / 256;
    if (g < 1) g = 1;
    if (g > device_sm_count() * 16) g = device_sm_count() * 16;
    use_max_smem(k_query);
    k_query<<<(int)g, 256, 0, st>>>(f, (const ulonglong2 *)keys128, n, out);
}

}  // namespace rsb
