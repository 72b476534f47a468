// pg_noalloc.cu -- pg_next_prime_noalloc: the persistent work-queue search
// of pg_search.cuh for caller-supplied numbers, with its working memory in a
// file-scope device array instead of memory the library allocates.
//
// Who needs it: callers that cannot call cudaMalloc (device memory owned by
// another allocator, or a running pipeline that must not stall on an
// allocation).  The caller passes device inputs and outputs; the queue head
// and the per-number "first probable prime" index live in g_noalloc_scratch.
//
// In host code g_noalloc_scratch names a host-side stand-in, not device
// memory: the host side passes the address cudaGetSymbolAddress returns for
// the current device, looked up once per device by the first call.
#include <cstdio>
#include <mutex>

#include "pg_internal.h"
#include "pg_limbs.h"
#include "pg_mont.cuh"

namespace pg {
namespace {

constexpr uint32_t NA_HEADER = 64;  // words before found[]: queue head (u64) and padding
constexpr uint32_t NA_WORDS = NA_HEADER + PG_NOALLOC_MAX_N;
constexpr int NA_MAX_DEVICES = 64;

// [0..1] queue head, [NA_HEADER .. NA_HEADER + n) first probable-prime step per number
static __device__ __align__(256) uint32_t g_noalloc_scratch[NA_WORDS];

// the first 64 odd primes, grouped so each group's product fits in 32 bits
__constant__ uint32_t c_group_prod[15] = {3234846615u, 95041567u,   907383479u, 4132280413u, 121330189u,
                                          257557397u,  490995677u,  842952707u, 1314423991u, 2125525169u,
                                          3073309843u, 16965341u,   20193023u,  23300239u,   29884301u};
__constant__ uint8_t c_group_len[15] = {9, 5, 5, 5, 4, 4, 4, 4, 4, 4, 4, 3, 3, 3, 3};
__constant__ uint16_t c_trial[64] = {3,   5,   7,   11,  13,  17,  19,  23,  29,  31,  37,  41,  43,
                                     47,  53,  59,  61,  67,  71,  73,  79,  83,  89,  97,  101, 103,
                                     107, 109, 113, 127, 131, 137, 139, 149, 151, 157, 163, 167, 173,
                                     179, 181, 191, 193, 197, 199, 211, 223, 227, 229, 233, 239, 241,
                                     251, 257, 263, 269, 271, 277, 281, 283, 293, 307, 311, 313};

// x + 2k as L words (x has `words` words, zero-extended).  Returns true when
// the sum carries out of word L-1, i.e. x + 2k does not fit in L words; the
// host picks L > words whenever a layout that wide exists, so this happens
// only for 48-word numbers within 2 * max_steps of 2^1536.
template <int L>
__device__ __forceinline__ bool load_plus(const uint32_t *__restrict__ row, uint32_t words, uint32_t k,
                                          uint32_t (&x)[L]) {
#pragma unroll
    for (int w = 0; w < L; w++) x[w] = ((uint32_t)w < words) ? row[w] : 0u;
    const uint64_t add = 2ull * k;
    x[0] = add_cc(x[0], (uint32_t)add);
    x[1] = addc_cc(x[1], (uint32_t)(add >> 32));
#pragma unroll
    for (int w = 2; w < L; w++) x[w] = addc_cc(x[w], 0u);
    return addc(0u, 0u) != 0u;
}

// true when x has a factor among the first 64 odd primes (and x is not that prime)
template <int L>
__device__ __forceinline__ bool trial_composite(const uint32_t (&x)[L]) {
    uint32_t hi = 0;
#pragma unroll
    for (int w = 1; w < L; w++) hi |= x[w];
    int pi = 0;
    for (int g = 0; g < 15; g++) {
        const uint32_t prod = c_group_prod[g];
        uint64_t r = 0;
#pragma unroll
        for (int w = L - 1; w >= 0; w--) r = ((r << 32) | x[w]) % prod;
        for (int t = 0; t < c_group_len[g]; t++, pi++) {
            const uint32_t q = c_trial[pi];
            if ((uint32_t)(r % q) == 0 && !(hi == 0 && x[0] == q)) return true;
        }
    }
    return false;
}

// Items t = k * n + i: the k-th odd candidate after number i, nearest first
// across all numbers.  Same queue, lane refill and atomicMin as
// k_search_persistent: a number's result is the smallest k that passed,
// because items are skipped only behind a smaller found k.
template <int L>
__global__ void __launch_bounds__(128) k_next_prime_noalloc(const uint32_t *__restrict__ nums, uint32_t n,
                                                            uint32_t words, unsigned long long total,
                                                            uint32_t *scratch) {
    const unsigned FULL = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31;
    unsigned long long *head = reinterpret_cast<unsigned long long *>(scratch);
    uint32_t *found = scratch + NA_HEADER;
    bool have = false, exhausted = false;
    uint32_t i = 0, k = 0;
    uint32_t x[L];
    while (true) {
        while (!exhausted) {
            const unsigned need = __ballot_sync(FULL, !have);
            if (need == 0) break;
            const int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) base = atomicAdd(head, (unsigned long long)__popc(need));
            base = __shfl_sync(FULL, base, leader);
            if (base >= total) {
                exhausted = true;
                break;
            }
            if (!have) {
                const unsigned long long t = base + __popc(need & ((1u << lane) - 1));
                if (t < total) {
                    k = (uint32_t)(t / n);
                    i = (uint32_t)(t - (unsigned long long)k * n);
                    if (*(volatile const uint32_t *)&found[i] >= k) {
                        const bool wrapped = load_plus<L>(nums + (size_t)i * words, words, k, x);
                        have = !wrapped && !trial_composite<L>(x);
                    }
                }
            }
        }
        if (!__any_sync(FULL, have)) break;
        if (have) {
            if (prp_rounds<L>(x, 1) == 1) atomicMin(&found[i], k);
            have = false;
        }
    }
}

__global__ void k_noalloc_copy_out(uint32_t n, const uint32_t *scratch, uint32_t *out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = scratch[NA_HEADER + i];
}

template <int L>
cudaError_t launch_noalloc(const uint32_t *nums, uint32_t n, uint32_t words, uint32_t max_steps, uint32_t *scratch,
                           uint32_t *out, int sms, cudaStream_t st) {
    int per = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_next_prime_noalloc<L>, 128, 0);
    if (e != cudaSuccess) return e;
    const int grid = sms * (per > 0 ? per : 1);
    k_next_prime_noalloc<L><<<grid, 128, 0, st>>>(nums, n, words, (unsigned long long)n * max_steps, scratch);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_noalloc_copy_out<<<(n + 255) / 256, 256, 0, st>>>(n, scratch, out);
    return cudaGetLastError();
}

std::mutex g_mu;
uint32_t *g_scratch_ptr[NA_MAX_DEVICES] = {};

int na_fail(int code, const char *msg, cudaError_t e = cudaSuccess) {
    char buf[256];
    if (e != cudaSuccess)
        snprintf(buf, sizeof buf, "pg_next_prime_noalloc: %s: %s", msg, cudaGetErrorString(e));
    else
        snprintf(buf, sizeof buf, "pg_next_prime_noalloc: %s", msg);
    set_error(buf);
    return code;
}

}  // namespace
}  // namespace pg

extern "C" int pg_next_prime_noalloc(const uint32_t *d_numbers, uint32_t n, uint32_t words, uint32_t max_steps,
                                     uint32_t *d_steps, void *stream) {
    using namespace pg;
    if (n == 0) return PG_OK;
    if (!d_numbers || !d_steps) return na_fail(PG_ERR_ARG, "NULL buffer");
    if (n > PG_NOALLOC_MAX_N) {
        char msg[128];
        snprintf(msg, sizeof msg, "n=%u exceeds the scratch capacity PG_NOALLOC_MAX_N=%u", n, (unsigned)PG_NOALLOC_MAX_N);
        return na_fail(PG_ERR_ARG, msg);
    }
    if (words == 0) return na_fail(PG_ERR_ARG, "words must be > 0");
    if (max_steps == 0) return na_fail(PG_ERR_ARG, "max_steps must be > 0");
    if (words > 48) return na_fail(PG_ERR_UNSUPPORTED, "words above the compiled limit of 48");
    // a layout with a spare word holds every x + 2k (2k < 2^33); only 48-word
    // numbers run without one, and their candidates past 2^1536 are skipped
    uint32_t L = words < 48 ? pick_limbs(words + 1) : 0;
    if (L == 0 || L > 48) L = pick_limbs(words);
    if (L == 0 || L > 48) return na_fail(PG_ERR_UNSUPPORTED, "words above the compiled limit of 48");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return na_fail(PG_ERR_CUDA, "cudaGetDevice", e);
    if (dev < 0 || dev >= NA_MAX_DEVICES) return na_fail(PG_ERR_UNSUPPORTED, "device index above 63");
    uint32_t *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_scratch_ptr[dev]) {  // once per device, with that device current
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) return na_fail(PG_ERR_CUDA, "cudaGetSymbolAddress", e);
            g_scratch_ptr[dev] = static_cast<uint32_t *>(p);
        }
        scratch = g_scratch_ptr[dev];
    }
    int sms = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return na_fail(PG_ERR_CUDA, "cudaDeviceGetAttribute", e);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the previous call's contents stay in the array: clear the queue head and found[]
    if ((e = cudaMemsetAsync(scratch, 0, NA_HEADER * sizeof(uint32_t), st)) != cudaSuccess)
        return na_fail(PG_ERR_CUDA, "clearing the queue head", e);
    if ((e = cudaMemsetAsync(scratch + NA_HEADER, 0xff, (size_t)n * sizeof(uint32_t), st)) != cudaSuccess)
        return na_fail(PG_ERR_CUDA, "clearing the results", e);
#define PG_CASE(nl) \
    if (L == nl) e = launch_noalloc<nl>(d_numbers, n, words, max_steps, scratch, d_steps, sms, st);
    PG_LIMB_LIST(PG_CASE)
#undef PG_CASE
    if (e != cudaSuccess) return na_fail(PG_ERR_CUDA, "kernel launch", e);
    return PG_OK;
}
