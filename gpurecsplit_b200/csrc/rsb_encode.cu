// Encoding on the device: Golomb-Rice descriptor stream and the double Elias-Fano index.
//
//   RiceBitVector::Builder   RiceBitVector.hpp:58-134 (appendFixed / appendUnaryAll)
//   bucket loop + sentinel   SIMDRecSplit.hpp:707-714, :810
//   DoubleEF constructor     DoubleEF.hpp:140-365 (FAST_CONSTRUCTION jump table :286-320)
//
// Per bucket the stream holds the fixed parts x & (2^g - 1) of all nodes in DFS pre-order,
// then their unary parts (x >> g zeros and a one). Buckets are independent, so every
// bucket's bit offset comes from a scan of per-bucket lengths and all buckets are written
// in parallel with atomicOr into a zeroed word array.
#include "rsb_kernels.cuh"

namespace rsb {

namespace {

constexpr uint64_t kLog2Q = 8, kQ = 1ull << kLog2Q;                 // DoubleEF.hpp:44-46,62-63
constexpr uint64_t kSuperQ = 1ull << 14, kSuperQMask = kSuperQ - 1;  // :65-66
constexpr uint64_t kSuperQSize = 1 + (kSuperQ / kQ) / 4;             // :68

__device__ __forceinline__ uint64_t warp_sum64(uint64_t v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    return v;
}
__device__ __forceinline__ uint64_t warp_excl64(uint64_t v) {
    const int lane = threadIdx.x & 31;
    uint64_t inc = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint64_t o = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= d) inc += o;
    }
    return inc - v;
}

// ORs the low `width` (<= 63) bits of v into the bit array at bit `pos`.
__device__ __forceinline__ void or_bits(uint64_t *words, uint64_t pos, uint64_t v, uint32_t width) {
    if (width == 0 || v == 0) return;
    const uint64_t w = pos / 64;
    const uint32_t sh = pos % 64;
    atomicOr((unsigned long long *)&words[w], (unsigned long long)(v << sh));
    if (sh + width > 64) atomicOr((unsigned long long *)&words[w + 1], (unsigned long long)(v >> (64 - sh)));
}

__global__ void k_bucket_bits(const uint64_t *node_base, uint64_t nb, NodeArrays nodes, DevTables tab, uint32_t *bits,
                              uint32_t *fixed_bits, DevStatus *status) {
    const int lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x / 32);
    for (uint64_t b = blockIdx.x * (uint64_t)(blockDim.x / 32) + (threadIdx.x >> 5); b < nb; b += warps) {
        const uint64_t n0 = node_base[b], n1 = node_base[b + 1];
        uint64_t tot = 0, fx = 0;
        bool bad = false;
        for (uint64_t j = n0 + lane; j < n1; j += 32) {
            uint64_t x = nodes.seed[j];
            if (x >= kSeedFailed) {  // failed or never searched: reported, and sized as 0
                bad = true;
                x = 0;
            }
            const uint32_t g = tab.memo[nodes.size[j]] >> 27;
            const uint32_t u = (uint32_t)(x >> g);  // the reference keeps x >> g in a uint32 vector
            fx += g;
            tot += g + (uint64_t)u + 1;
        }
        if (bad) set_error(status, RSB_ERR_SEARCH_BUDGET, b);
        tot = warp_sum64(tot);
        fx = warp_sum64(fx);
        if (lane == 0) {
            bits[b] = (uint32_t)tot;
            fixed_bits[b] = (uint32_t)fx;
        }
    }
}

__global__ void k_write_rice(const uint64_t *node_base, uint64_t nb, NodeArrays nodes, DevTables tab,
                             const uint64_t *pos_acc, const uint32_t *fixed_bits, uint64_t *desc, uint64_t cap_words,
                             EfParams *ef, DevStatus *status) {
    // A build that already failed (a search without a seed, a duplicate key, ...) writes
    // nothing: its seeds are not codes, and the unary part of an unfound seed would land
    // outside the stream.
    if (*(const volatile int *)&status->code) return;
    const uint64_t total = pos_acc[nb];
    const uint64_t words = (((total + 1 + 7) / 8) + 7 + 7) / 8;  // resize rule of appendFixed, :77
    if (words > cap_words) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_error(status, RSB_ERR_INTERNAL, words);
        return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ef->total_bits = total;
        ef->desc_words = words;
        atomicOr((unsigned long long *)&desc[total / 64], 1ull << (total % 64));  // sentinel appendFixed(1, 1)
    }
    const int lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x / 32);
    for (uint64_t b = blockIdx.x * (uint64_t)(blockDim.x / 32) + (threadIdx.x >> 5); b < nb; b += warps) {
        const uint64_t n0 = node_base[b], n1 = node_base[b + 1];
        uint64_t fpos = pos_acc[b];
        uint64_t upos = fpos + fixed_bits[b];
        for (uint64_t j0 = n0; j0 < n1; j0 += 32) {
            const uint64_t j = j0 + lane;
            const bool valid = j < n1;
            uint64_t x = 0;
            uint32_t g = 0, u1 = 0;
            if (valid) {
                x = nodes.seed[j];
                g = tab.memo[nodes.size[j]] >> 27;
                u1 = (uint32_t)(x >> g) + 1;
            }
            const uint64_t ge = warp_excl64(g), ue = warp_excl64(u1);
            if (valid) {
                or_bits(desc, fpos + ge, x & ((1ull << g) - 1), g);
                const uint64_t one = upos + ue + u1 - 1;
                atomicOr((unsigned long long *)&desc[one / 64], 1ull << (one % 64));
            }
            fpos += warp_sum64(g);
            upos += warp_sum64(u1);
        }
    }
}

// ---- double Elias-Fano ----------------------------------------------------------------

__device__ __forceinline__ uint64_t bpk_of(const uint64_t *cum, const uint64_t *pos, uint64_t nb) {
    // DoubleEF.hpp:144, the single floating-point operation of the path (IEEE double).
    // With no keys the reference divides 0 by 0 and converts the NaN to uint64; on its x86-64
    // build that conversion yields 0x8000000000000000, which is what is stored here.
    if (cum[nb] == 0) return 1ull << 63;
    return (uint64_t)((double)(1ull << 20) * ((double)pos[nb] / (double)cum[nb]));
}

__global__ void k_ef_init(const uint64_t *cum, const uint64_t *pos, uint64_t nb, EfParams *ef) {
    if (threadIdx.x == 0) {
        ef->num_buckets = nb;
        ef->bits_per_key_fixed_point = bpk_of(cum, pos, nb);
        ef->cum_keys_min_delta = INT64_MAX / 2;
        ef->min_diff = INT64_MAX / 2;
    }
}

__global__ void k_ef_reduce(const uint64_t *cum, const uint64_t *pos, uint64_t nb, EfParams *ef) {
    const uint64_t bpk = ef->bits_per_key_fixed_point;
    int64_t md = INT64_MAX / 2, mdiff = INT64_MAX / 2;
    for (uint64_t i = 1 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= nb; i += (uint64_t)gridDim.x * blockDim.x) {
        md = min(md, (int64_t)(cum[i] - cum[i - 1]));
        const int64_t bb = (int64_t)pos[i] - (int64_t)(bpk * cum[i] >> 20);
        const int64_t bp = (int64_t)pos[i - 1] - (int64_t)(bpk * cum[i - 1] >> 20);
        mdiff = min(mdiff, bb - bp);
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        md = min(md, (int64_t)__shfl_xor_sync(0xffffffffu, (long long)md, d));
        mdiff = min(mdiff, (int64_t)__shfl_xor_sync(0xffffffffu, (long long)mdiff, d));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin((long long *)&ef->cum_keys_min_delta, (long long)md);
        atomicMin((long long *)&ef->min_diff, (long long)mdiff);
    }
}

__device__ __forceinline__ uint64_t lambda64(uint64_t w) { return 63 - __clzll(w); }

__global__ void k_ef_params(const uint64_t *cum, const uint64_t *pos, uint64_t nb, EfParams *ef, uint64_t lower_cap,
                            uint64_t cum_cap, uint64_t pos_cap, uint64_t jump_cap, DevStatus *status) {
    if (threadIdx.x != 0) return;
    const uint64_t bpk = ef->bits_per_key_fixed_point;
    const int64_t md = ef->cum_keys_min_delta, mdiff = ef->min_diff;
    // DoubleEF.hpp:181-185
    ef->u_position = (uint64_t)((int64_t)pos[nb] - (int64_t)(bpk * cum[nb] >> 20) - (int64_t)(nb * mdiff) + 1);
    ef->l_position = ef->u_position / (nb + 1) == 0 ? 0 : lambda64(ef->u_position / (nb + 1));
    ef->u_cum_keys = cum[nb] - nb * md + 1;
    ef->l_cum_keys = ef->u_cum_keys / (nb + 1) == 0 ? 0 : lambda64(ef->u_cum_keys / (nb + 1));
    // :88-95
    ef->lower_words = ((nb + 1) * (ef->l_cum_keys + ef->l_position) + 63) / 64 + 1;
    ef->cum_words = (nb + 1 + (ef->u_cum_keys >> ef->l_cum_keys) + 63) / 64;
    ef->pos_words = (nb + 1 + (ef->u_position >> ef->l_position) + 63) / 64;
    uint64_t jw = (nb / kSuperQ) * kSuperQSize * 2;
    if (nb % kSuperQ != 0) jw += (1 + ((nb % kSuperQ + kQ - 1) / kQ + 3) / 4) * 2;
    ef->jump_words = jw;
    if (ef->l_cum_keys * 2 + ef->l_position > 56 || ef->lower_words > lower_cap || ef->cum_words > cum_cap ||
        ef->pos_words > pos_cap || jw > jump_cap)
        set_error(status, RSB_ERR_INTERNAL, 1);
}

__global__ void k_ef_fill(const uint64_t *cum, const uint64_t *pos, uint64_t nb, const EfParams *efp, uint64_t *lower,
                          uint64_t *upper_cum, uint64_t *upper_pos, uint64_t *jump, const DevStatus *status) {
    if (*(const volatile int *)&status->code) return;
    const EfParams ef = *efp;
    const uint64_t lc = ef.l_cum_keys, lp = ef.l_position;
    const uint64_t mc = (1ull << lc) - 1, mp = (1ull << lp) - 1;
    const uint64_t md = (uint64_t)ef.cum_keys_min_delta, mdiff = (uint64_t)ef.min_diff;
    const uint64_t bpk = ef.bits_per_key_fixed_point;
    auto cum_val = [&](uint64_t i) { return cum[i] - i * md; };
    auto pos_val = [&](uint64_t i) { return (uint64_t)((int64_t)pos[i] - (int64_t)(bpk * cum[i] >> 20)) - i * mdiff; };
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= nb; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t cv = cum_val(i), pv = pos_val(i);
        // lower bits: [cum low lc bits | position low lp bits] at i * (lc + lp), DoubleEF.hpp:275-279
        or_bits(lower, i * (lc + lp), (cv & mc) | ((pv & mp) << lc), (uint32_t)(lc + lp));
        const uint64_t pc = (cv >> lc) + i, pp = (pv >> lp) + i;  // :276, :280
        atomicOr((unsigned long long *)&upper_cum[pc / 64], 1ull << (pc % 64));
        atomicOr((unsigned long long *)&upper_pos[pp / 64], 1ull << (pp % 64));
        // Entry i is the i-th one of each upper-bit array (positions strictly increase), so
        // the jump table of :288-320 needs no select: every q-th entry stores its own position.
        if ((i & (kQ - 1)) == 0) {
            const uint64_t blk = (i / kSuperQ) * (kSuperQSize * 2);
            const uint64_t i0 = i - (i & kSuperQMask);
            const uint64_t pc0 = (cum_val(i0) >> lc) + i0, pp0 = (pos_val(i0) >> lp) + i0;
            if ((i & kSuperQMask) == 0) {
                if (blk < ef.jump_words) jump[blk] = pc;
                if (blk + 1 < ef.jump_words) jump[blk + 1] = pp;
            }
            const uint64_t slot = 2 * ((i & kSuperQMask) / kQ);
            if (blk + 2 + slot / 4 < ef.jump_words) {
                uint16_t *j16 = (uint16_t *)(jump + blk + 2);
                j16[slot] = (uint16_t)(pc - pc0);
                j16[slot + 1] = (uint16_t)(pp - pp0);
            }
        }
    }
}

// Algorithmic work of the searches: sum over nodes of (candidates up to the found seed) * m,
// candidates being seeds (splits, brute-force leaves) or rotation bases (rotation leaves).
// Nodes of the four search stages (almost all nodes) sum in registers and then per warp, so
// that a block's threads do not all contend for the same few shared-memory counters; the
// fanout-2 stages add to shared memory directly.
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void k_evals(const uint64_t *node_total, NodeArrays nodes, uint32_t leaf, uint32_t rotate, EfParams *ef,
                        uint64_t *windows) {
    constexpr int kSearch = kNumStages - kStageUpper;  // stages kStageUpper .. kNumStages - 1
    __shared__ unsigned long long s_acc[kNumStages], s_win[kNumStages];
    for (int s = threadIdx.x; s < kNumStages; s += blockDim.x) s_acc[s] = s_win[s] = 0;
    __syncthreads();
    unsigned long long acc[kSearch], win[kSearch];
#pragma unroll
    for (int k = 0; k < kSearch; ++k) acc[k] = win[k] = 0;
    const uint64_t n = *node_total;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t x = nodes.seed[j];
        const uint32_t m = nodes.size[j];
        const uint32_t stage = nodes.stage[j];
        const bool ok = x < kSeedFailed;
        const uint64_t trials = (rotate && m == leaf) ? x / leaf + 1 : x + 1;
        const unsigned long long work = ok ? (unsigned long long)(trials * m) : 0ull;
        if (stage >= (uint32_t)kStageUpper) {
            const unsigned long long w = nodes.next_win[j];
#pragma unroll
            for (int k = 0; k < kSearch; ++k)
                if (stage == (uint32_t)(kStageUpper + k)) {
                    acc[k] += work;
                    win[k] += w;
                }
        } else if (ok) {
            atomicAdd(&s_acc[stage], work);
        }
    }
#pragma unroll
    for (int k = 0; k < kSearch; ++k) {
        acc[k] = warp_sum_u64(acc[k]);
        win[k] = warp_sum_u64(win[k]);
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < kSearch; ++k) {
            if (acc[k]) atomicAdd(&s_acc[kStageUpper + k], acc[k]);
            if (win[k]) atomicAdd(&s_win[kStageUpper + k], win[k]);
        }
    }
    __syncthreads();
    for (int s = threadIdx.x; s < kNumStages; s += blockDim.x) {
        if (s_acc[s]) {
            atomicAdd((unsigned long long *)&ef->evals_stage[s], s_acc[s]);
            atomicAdd((unsigned long long *)&ef->evals_alg, s_acc[s]);
        }
        if (s_win[s]) atomicAdd((unsigned long long *)&windows[s], s_win[s]);
    }
}

int grid_for(uint64_t n, int threads, int cap) {
    uint64_t g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > (uint64_t)cap) g = cap;
    return (int)g;
}

}  // namespace

void launch_bucket_bits(const uint64_t *node_base, uint64_t nb, NodeArrays nodes, DevTables tab, uint32_t *bits,
                        uint32_t *fixed_bits, DevStatus *status, cudaStream_t st) {
    use_max_smem(k_bucket_bits);
    k_bucket_bits<<<grid_for(nb * 32, 256, device_sm_count() * 8), 256, 0, st>>>(node_base, nb, nodes, tab, bits, fixed_bits, status);
    count_launches(1);
}

void launch_write_rice(const uint64_t *node_base, uint64_t nb, NodeArrays nodes, DevTables tab, const uint64_t *pos_acc,
                       const uint32_t *fixed_bits, uint64_t *desc, uint64_t desc_cap_words, EfParams *ef,
                       DevStatus *status, cudaStream_t st) {
    use_max_smem(k_write_rice);
    k_write_rice<<<grid_for(nb * 32, 256, device_sm_count() * 8), 256, 0, st>>>(node_base, nb, nodes, tab, pos_acc, fixed_bits, desc,
                                                                   desc_cap_words, ef, status);
    count_launches(1);
}

void launch_ef_build(const uint64_t *cum, const uint64_t *pos, uint64_t nb, uint64_t /*keys*/, EfParams *ef,
                     uint64_t *lower, uint64_t lower_cap, uint64_t *upper_cum, uint64_t cum_cap, uint64_t *upper_pos,
                     uint64_t pos_cap, uint64_t *jump, uint64_t jump_cap, DevStatus *status, cudaStream_t st) {
    use_max_smem(k_ef_init);
    k_ef_init<<<1, 32, 0, st>>>(cum, pos, nb, ef);
    use_max_smem(k_ef_reduce);
    k_ef_reduce<<<grid_for(nb, 256, device_sm_count() * 4), 256, 0, st>>>(cum, pos, nb, ef);
    use_max_smem(k_ef_params);
    k_ef_params<<<1, 32, 0, st>>>(cum, pos, nb, ef, lower_cap, cum_cap, pos_cap, jump_cap, status);
    use_max_smem(k_ef_fill);
    k_ef_fill<<<grid_for(nb + 1, 256, device_sm_count() * 8), 256, 0, st>>>(cum, pos, nb, ef, lower, upper_cum, upper_pos, jump, status);
    count_launches(4);
}

void launch_evals(const uint64_t *node_total, NodeArrays nodes, uint32_t leaf, uint32_t rotate, EfParams *ef,
                  uint64_t *windows, cudaStream_t st) {
    use_max_smem(k_evals);
    k_evals<<<device_sm_count() * 4, 256, 0, st>>>(node_total, nodes, leaf, rotate, ef, windows);
    count_launches(1);
}

}  // namespace rsb
