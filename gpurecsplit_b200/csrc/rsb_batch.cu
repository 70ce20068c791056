// Set-aware kernels of the batched construction: many independent key sets in one pipeline.
//
// Set s owns keys [set_key[s], set_key[s+1]) and buckets [set_bucket[s], set_bucket[s+1]),
// with max(1, ceil(n_s / b)) buckets as a plain build of that set has. A key's bucket is
// set_bucket[s] + remap128(first, nb_s) (AbstractParallelRecSplit.hpp:322), so the global
// bucket order keeps every set's keys contiguous and in its own bucket order. Tree emission,
// stage lists and every seed search then run over the global buckets unchanged. Each set
// gets its own Golomb-Rice stream (starting at bit 0 of its own word vector, sentinel after
// its last bucket) and its own double Elias-Fano index, exactly as its plain build would.
#include "rsb_kernels.cuh"
#include "rsb_partition.cuh"

namespace rsb {

namespace {

constexpr uint64_t kQ = 256, kSuperQ = 1ull << 14, kSuperQMask = kSuperQ - 1;
constexpr uint64_t kSuperQSize = 1 + (kSuperQ / kQ) / 4;

int grid_for(uint64_t n, int threads, int cap) {
    uint64_t g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > (uint64_t)cap) g = cap;
    return (int)g;
}

// Largest s with a[s] <= v among a[0..n] (a non-decreasing, a[0] <= v).
__device__ __forceinline__ uint32_t upper_index(const uint64_t *a, uint32_t n, uint64_t v) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (a[mid] <= v) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void k_set_nbuckets(const uint64_t *set_key, uint32_t nsets, uint64_t bucket_size, uint32_t *nb) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < nsets; s += gridDim.x * blockDim.x) {
        const uint64_t n = set_key[s + 1] - set_key[s];
        const uint64_t b = (n + bucket_size - 1) / bucket_size;  // SIMDRecSplit.hpp:774
        nb[s] = (uint32_t)(b < 1 ? 1 : b);
    }
}

// Bucket ids of a batched build, counted per bucket. Keys are taken in contiguous chunks of
// kPartChunk per CTA, so a chunk spans few sets: its set range is found once, each key
// searches only inside it, and when the chunk's buckets fit kPartBins the counts are
// gathered in shared memory and flushed with one global atomic per non-empty bucket.
__global__ void __launch_bounds__(kPartThreads) k_set_bucket_ids(const ulonglong2 *__restrict__ keys, uint64_t n,
                                                                  const uint64_t *set_key, const uint64_t *set_bucket,
                                                                  uint32_t nsets, uint32_t *bucket_id, uint32_t *counts) {
    __shared__ uint32_t bins[kPartBins];
    __shared__ uint32_t s_lo, s_hi;
    for (uint64_t c0 = (uint64_t)blockIdx.x * kPartChunk; c0 < n; c0 += (uint64_t)gridDim.x * kPartChunk) {
        const uint64_t c1 = c0 + kPartChunk < n ? c0 + kPartChunk : n;
        __syncthreads();
        if (threadIdx.x == 0) {
            // sets may be empty: a key belongs to the last set whose first key is <= it
            s_lo = upper_index(set_key, nsets, c0);
            s_hi = upper_index(set_key, nsets, c1 - 1);
        }
        __syncthreads();
        const uint32_t lo = s_lo, hi = s_hi;
        const uint64_t b0 = set_bucket[lo], nbins = set_bucket[hi + 1] - b0;
        const bool local = nbins <= kPartBins;
        if (local)
            for (uint32_t j = threadIdx.x; j < nbins; j += kPartThreads) bins[j] = 0;
        __syncthreads();
        for (uint64_t i = c0 + threadIdx.x; i < c1; i += kPartThreads) {
            uint32_t s = lo;
            if (hi != lo) s = lo + upper_index(set_key + lo, hi - lo + 1, i);
            const uint64_t nb = set_bucket[s + 1] - set_bucket[s];
            const uint32_t b = (uint32_t)(set_bucket[s] + remap128(keys[i].x, nb));
            bucket_id[i] = b;
            if (local) atomicAdd(&bins[b - b0], 1u);
            else atomicAdd(&counts[b], 1u);
        }
        __syncthreads();
        if (local)
            for (uint32_t j = threadIdx.x; j < nbins; j += kPartThreads)
                if (bins[j]) atomicAdd(&counts[b0 + j], bins[j]);
    }
}

// Descriptor words of each set: the appendFixed resize rule applied after its sentinel.
__global__ void k_set_desc_words(const uint64_t *pos_acc, const uint64_t *set_bucket, uint32_t nsets, uint32_t *words,
                                 uint64_t *set_bits) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < nsets; s += gridDim.x * blockDim.x) {
        const uint64_t bits = pos_acc[set_bucket[s + 1]] - pos_acc[set_bucket[s]];
        set_bits[s] = bits;
        words[s] = (uint32_t)((((bits + 1 + 7) / 8) + 7 + 7) / 8);
    }
}

__device__ __forceinline__ void or_bits(uint64_t *w, uint64_t pos, uint64_t v, uint32_t width) {
    if (width == 0 || v == 0) return;
    const uint64_t k = pos / 64;
    const uint32_t sh = pos % 64;
    atomicOr((unsigned long long *)&w[k], (unsigned long long)(v << sh));
    if (sh + width > 64) atomicOr((unsigned long long *)&w[k + 1], (unsigned long long)(v >> (64 - sh)));
}

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

// Rice writer over all sets: one warp per global bucket writes at the bucket's offset
// inside its own set's stream; lane 0 of each set's first bucket writes the sentinel.
__global__ void k_set_write_rice(const uint64_t *node_base, uint64_t nb_total, NodeArrays nodes, DevTables tab,
                                 const uint64_t *pos_acc, const uint32_t *fixed_bits, const uint64_t *set_bucket,
                                 uint32_t nsets, const uint64_t *word_base, const uint64_t *set_bits, uint64_t *desc,
                                 uint64_t cap_words, DevStatus *status) {
    // A failed build writes nothing (its unfound seeds are not codes; see k_write_rice).
    if (*(const volatile int *)&status->code) return;
    if (word_base[nsets] > cap_words) {  // would overflow the output buffer: report instead
        if (blockIdx.x == 0 && threadIdx.x == 0) set_error(status, RSB_ERR_INTERNAL, word_base[nsets]);
        return;
    }
    const int lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x / 32);
    for (uint64_t b = blockIdx.x * (uint64_t)(blockDim.x / 32) + (threadIdx.x >> 5); b < nb_total; b += warps) {
        const uint32_t s = upper_index(set_bucket, nsets, b);
        uint64_t *d = desc + word_base[s];
        const uint64_t base_bit = pos_acc[set_bucket[s]];
        if (b == set_bucket[s] && lane == 0) {
            const uint64_t t = set_bits[s];
            atomicOr((unsigned long long *)&d[t / 64], 1ull << (t % 64));  // sentinel appendFixed(1, 1)
        }
        const uint64_t n0 = node_base[b], n1 = node_base[b + 1];
        uint64_t fpos = pos_acc[b] - base_bit;
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
                or_bits(d, fpos + ge, x & ((1ull << g) - 1), g);
                const uint64_t one = upos + ue + u1 - 1;
                atomicOr((unsigned long long *)&d[one / 64], 1ull << (one % 64));
            }
            fpos += warp_sum64(g);
            upos += warp_sum64(u1);
        }
    }
}

// ---- per-set double Elias-Fano (one CTA per set) ----------------------------------------
constexpr int kEfThreads = 256;

struct SetView {
    const uint64_t *acc, *pos;  // global bucket_size_acc / bucket_pos_acc
    uint64_t b0, nb, key0, pos0;
    __device__ uint64_t cum(uint64_t i) const { return acc[b0 + i] - key0; }
    __device__ uint64_t position(uint64_t i) const { return pos[b0 + i] - pos0; }
};

__device__ SetView set_view(const uint64_t *acc, const uint64_t *pos, const uint64_t *set_bucket, uint32_t s) {
    SetView v;
    v.acc = acc;
    v.pos = pos;
    v.b0 = set_bucket[s];
    v.nb = set_bucket[s + 1] - v.b0;
    v.key0 = acc[v.b0];
    v.pos0 = pos[v.b0];
    return v;
}

__device__ __forceinline__ uint64_t lambda64(uint64_t w) { return 63 - __clzll(w); }

template <typename T, typename Op>
__device__ T block_reduce(T v, Op op, T *scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v = op(v, (T)__shfl_xor_sync(0xffffffffu, (long long)v, d));
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < kEfThreads / 32 ? scratch[lane] : scratch[0];
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) v = op(v, (T)__shfl_xor_sync(0xffffffffu, (long long)v, d));
        if (lane == 0) scratch[0] = v;
    }
    __syncthreads();
    const T r = scratch[0];
    __syncthreads();
    return r;
}

// DoubleEF.hpp:140-185 per set: bits_per_key_fixed_point, minimum deltas, u and l.
__global__ void __launch_bounds__(kEfThreads) k_set_ef_params(const uint64_t *acc, const uint64_t *pos,
                                                              const uint64_t *set_bucket, uint32_t nsets, EfParams *ef,
                                                              uint32_t *lower_w, uint32_t *cum_w, uint32_t *pos_w,
                                                              uint32_t *jump_w) {
    __shared__ long long scratch[kEfThreads / 32];
    const uint32_t s = blockIdx.x;
    if (s >= nsets) return;
    const SetView v = set_view(acc, pos, set_bucket, s);
    const uint64_t nb = v.nb;
    const uint64_t nkeys = v.cum(nb), nbits = v.position(nb);
    // no keys: 0/0 in the reference, whose x86-64 build turns the NaN into 0x8000000000000000
    const uint64_t bpk = nkeys == 0 ? (1ull << 63) : (uint64_t)((double)(1ull << 20) * ((double)nbits / (double)nkeys));
    long long md = INT64_MAX / 2, mdiff = INT64_MAX / 2;
    for (uint64_t i = 1 + threadIdx.x; i <= nb; i += kEfThreads) {
        md = min(md, (long long)(v.cum(i) - v.cum(i - 1)));
        const long long bb = (long long)v.position(i) - (long long)(bpk * v.cum(i) >> 20);
        const long long bp = (long long)v.position(i - 1) - (long long)(bpk * v.cum(i - 1) >> 20);
        mdiff = min(mdiff, bb - bp);
    }
    auto mn = [](long long a, long long b) { return a < b ? a : b; };
    md = block_reduce<long long>(md, mn, scratch);
    mdiff = block_reduce<long long>(mdiff, mn, scratch);
    if (threadIdx.x == 0) {
        EfParams p{};
        p.num_buckets = nb;
        p.bits_per_key_fixed_point = bpk;
        p.cum_keys_min_delta = md;
        p.min_diff = mdiff;
        p.u_position = (uint64_t)((int64_t)nbits - (int64_t)(bpk * nkeys >> 20) - (int64_t)(nb * mdiff) + 1);
        p.l_position = p.u_position / (nb + 1) == 0 ? 0 : lambda64(p.u_position / (nb + 1));
        p.u_cum_keys = nkeys - nb * md + 1;
        p.l_cum_keys = p.u_cum_keys / (nb + 1) == 0 ? 0 : lambda64(p.u_cum_keys / (nb + 1));
        p.lower_words = ((nb + 1) * (p.l_cum_keys + p.l_position) + 63) / 64 + 1;
        p.cum_words = (nb + 1 + (p.u_cum_keys >> p.l_cum_keys) + 63) / 64;
        p.pos_words = (nb + 1 + (p.u_position >> p.l_position) + 63) / 64;
        uint64_t jw = (nb / kSuperQ) * kSuperQSize * 2;
        if (nb % kSuperQ != 0) jw += (1 + ((nb % kSuperQ + kQ - 1) / kQ + 3) / 4) * 2;
        p.jump_words = jw;
        p.total_bits = nbits;
        p.desc_words = (((nbits + 1 + 7) / 8) + 7 + 7) / 8;
        ef[s] = p;
        lower_w[s] = (uint32_t)p.lower_words;
        cum_w[s] = (uint32_t)p.cum_words;
        pos_w[s] = (uint32_t)p.pos_words;
        jump_w[s] = (uint32_t)jw;
    }
}

// DoubleEF.hpp:266-320 per set (entries are written with atomicOr into zeroed arrays).
__global__ void __launch_bounds__(kEfThreads) k_set_ef_fill(const uint64_t *acc, const uint64_t *pos,
                                                            const uint64_t *set_bucket, uint32_t nsets, const EfParams *ef,
                                                            const uint64_t *lower_base, const uint64_t *cum_base,
                                                            const uint64_t *pos_base, const uint64_t *jump_base,
                                                            uint64_t *lower, uint64_t *upper_cum, uint64_t *upper_pos,
                                                            uint64_t *jump) {
    const uint32_t s = blockIdx.x;
    if (s >= nsets) return;
    const SetView v = set_view(acc, pos, set_bucket, s);
    const EfParams p = ef[s];
    uint64_t *lw = lower + lower_base[s], *uc = upper_cum + cum_base[s], *up = upper_pos + pos_base[s];
    uint64_t *jp = jump + jump_base[s];
    const uint64_t lc = p.l_cum_keys, lp = p.l_position;
    const uint64_t mc = (1ull << lc) - 1, mp = (1ull << lp) - 1;
    const uint64_t md = (uint64_t)p.cum_keys_min_delta, mdiff = (uint64_t)p.min_diff, bpk = p.bits_per_key_fixed_point;
    auto cum_val = [&](uint64_t i) { return v.cum(i) - i * md; };
    auto pos_val = [&](uint64_t i) { return (uint64_t)((int64_t)v.position(i) - (int64_t)(bpk * v.cum(i) >> 20)) - i * mdiff; };
    for (uint64_t i = threadIdx.x; i <= v.nb; i += kEfThreads) {
        const uint64_t cv = cum_val(i), pv = pos_val(i);
        or_bits(lw, i * (lc + lp), (cv & mc) | ((pv & mp) << lc), (uint32_t)(lc + lp));
        const uint64_t pc = (cv >> lc) + i, pp = (pv >> lp) + i;
        atomicOr((unsigned long long *)&uc[pc / 64], 1ull << (pc % 64));
        atomicOr((unsigned long long *)&up[pp / 64], 1ull << (pp % 64));
        if ((i & (kQ - 1)) == 0) {
            const uint64_t blk = (i / kSuperQ) * (kSuperQSize * 2);
            const uint64_t i0 = i - (i & kSuperQMask);
            const uint64_t pc0 = (cum_val(i0) >> lc) + i0, pp0 = (pos_val(i0) >> lp) + i0;
            if ((i & kSuperQMask) == 0) {
                if (blk < p.jump_words) jp[blk] = pc;
                if (blk + 1 < p.jump_words) jp[blk + 1] = pp;
            }
            const uint64_t slot = 2 * ((i & kSuperQMask) / kQ);
            if (blk + 2 + slot / 4 < p.jump_words) {
                uint16_t *j16 = (uint16_t *)(jp + blk + 2);
                j16[slot] = (uint16_t)(pc - pc0);
                j16[slot + 1] = (uint16_t)(pp - pp0);
            }
        }
    }
}

}  // namespace

void launch_set_nbuckets(const uint64_t *set_key, uint32_t nsets, uint64_t bucket_size, uint32_t *nb, cudaStream_t st) {
    use_max_smem(k_set_nbuckets);
    k_set_nbuckets<<<grid_for(nsets, 256, 1024), 256, 0, st>>>(set_key, nsets, bucket_size, nb);
    count_launches(1);
}

void launch_set_bucket_ids(const uint64_t *keys128, uint64_t n, const uint64_t *set_key, const uint64_t *set_bucket,
                           uint32_t nsets, uint64_t nb_total, uint32_t *bucket_id, uint32_t *counts, cudaStream_t st) {
    cudaMemsetAsync(counts, 0, nb_total * sizeof(uint32_t), st);
    use_max_smem(k_set_bucket_ids);
    k_set_bucket_ids<<<grid_for(n, kPartChunk, device_sm_count() * 6), kPartThreads, 0, st>>>((const ulonglong2 *)keys128, n, set_key,
                                                                                set_bucket, nsets, bucket_id, counts);
    count_launches(1);
}

void launch_set_scatter(const uint64_t *keys128, uint64_t n, const uint64_t *set_key, const uint64_t *set_bucket,
                        uint32_t nsets, const uint32_t *bucket_id, const uint64_t *acc, uint32_t *cursor,
                        uint64_t nb_total, uint64_t *sorted, cudaStream_t st) {
    cudaMemsetAsync(cursor, 0, nb_total * sizeof(uint32_t), st);
    const SetBuckets map{set_key, set_bucket, nsets, bucket_id};
    use_max_smem(k_chunk_scatter<SetBuckets>);
    k_chunk_scatter<<<grid_for(n, kPartChunk, device_sm_count() * 6), kPartThreads, 0, st>>>((const ulonglong2 *)keys128, n, map, acc,
                                                                               cursor, sorted);
    count_launches(1);
}

void launch_set_desc_words(const uint64_t *pos_acc, const uint64_t *set_bucket, uint32_t nsets, uint32_t *words,
                           uint64_t *set_bits, cudaStream_t st) {
    use_max_smem(k_set_desc_words);
    k_set_desc_words<<<grid_for(nsets, 256, 1024), 256, 0, st>>>(pos_acc, set_bucket, nsets, words, set_bits);
    count_launches(1);
}

void launch_set_write_rice(const uint64_t *node_base, uint64_t nb_total, NodeArrays nodes, DevTables tab,
                           const uint64_t *pos_acc, const uint32_t *fixed_bits, const uint64_t *set_bucket,
                           uint32_t nsets, const uint64_t *word_base, const uint64_t *set_bits, uint64_t *desc,
                           uint64_t cap_words, DevStatus *status, cudaStream_t st) {
    use_max_smem(k_set_write_rice);
    k_set_write_rice<<<grid_for(nb_total * 32, 256, device_sm_count() * 8), 256, 0, st>>>(node_base, nb_total, nodes, tab, pos_acc,
                                                                          fixed_bits, set_bucket, nsets, word_base,
                                                                          set_bits, desc, cap_words, status);
    count_launches(1);
}

void launch_set_ef_params(const uint64_t *acc, const uint64_t *pos, const uint64_t *set_bucket, uint32_t nsets,
                          EfParams *ef, uint32_t *lower_w, uint32_t *cum_w, uint32_t *pos_w, uint32_t *jump_w,
                          cudaStream_t st) {
    if (nsets == 0) return;
    use_max_smem(k_set_ef_params);
    k_set_ef_params<<<nsets, kEfThreads, 0, st>>>(acc, pos, set_bucket, nsets, ef, lower_w, cum_w, pos_w, jump_w);
    count_launches(1);
}

void launch_set_ef_fill(const uint64_t *acc, const uint64_t *pos, const uint64_t *set_bucket, uint32_t nsets,
                        const EfParams *ef, const uint64_t *lower_base, const uint64_t *cum_base, const uint64_t *pos_base,
                        const uint64_t *jump_base, uint64_t *lower, uint64_t *upper_cum, uint64_t *upper_pos,
                        uint64_t *jump, cudaStream_t st) {
    if (nsets == 0) return;
    use_max_smem(k_set_ef_fill);
    k_set_ef_fill<<<nsets, kEfThreads, 0, st>>>(acc, pos, set_bucket, nsets, ef, lower_base, cum_base, pos_base,
                                                jump_base, lower, upper_cum, upper_pos, jump);
    count_launches(1);
}

}  // namespace rsb
