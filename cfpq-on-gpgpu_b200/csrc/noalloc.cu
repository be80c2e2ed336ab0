// cfpq_hash_count_rows_noalloc: the result hash / count of a CFPQ answer
// matrix that the caller keeps in its own device memory, computed without
// allocating anything.
//
// Who it is for: callers that cannot call cudaMalloc.  Some hosts hand all
// device memory to their own pool allocator at start-up (a cudaMalloc from
// this library would then fail or compete with that pool), and some
// latency-sensitive serving loops cannot accept the implicit device-wide
// synchronisation a cudaMalloc / cudaFree may cause.  Such callers pass the
// matrix and a small output buffer that they allocated themselves.
//
// The scratch memory the hash needs (the 11^(n-1-c) and 13^(n-1-r) power
// tables and two 64-bit accumulators) lives in the file-scope device array
// `g_noalloc_scratch` below, sized for n <= CFPQ_NOALLOC_MAX_N.  Every GPU
// that loads this library holds that array (about 512 KiB) until the process
// exits.  All calls on one device share it and it keeps the last call's
// contents: every call rebuilds the power tables and clears the accumulators
// before use, and calls whose work overlaps on the GPU (for example on two
// streams without ordering) race on the array and give wrong results.  The
// array's address is looked up per device and CUDA context: a first call in
// a new context (after cudaDeviceReset, or under a caller's own driver
// context) repeats the set-up, so it too should come before any stream
// capture.
#include <cstdio>
#include <mutex>

#include "cfpq_b200.h"
#include "common.cuh"

namespace {

constexpr unsigned long long kMod = 1000000007ULL;  // cfpq-cpp/Grammar.cpp:14
constexpr uint32_t kMaxN = CFPQ_NOALLOC_MAX_N;
constexpr int kMaxDevices = 64;

// Layout: [0, 2) accumulators (hash terms, bit count) as unsigned long long,
// then pow11[kMaxN] and pow13[kMaxN] as uint32.
constexpr size_t kScratchBytes = 2 * sizeof(unsigned long long) + 2 * (size_t)kMaxN * sizeof(uint32_t);
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct ScratchView {
    unsigned long long *acc;  // [0] hash terms, [1] bit count
    uint32_t *pow11;
    uint32_t *pow13;
};

__host__ __device__ inline ScratchView view(void *base) {
    ScratchView v;
    v.acc = reinterpret_cast<unsigned long long *>(base);
    v.pow11 = reinterpret_cast<uint32_t *>(v.acc + 2);
    v.pow13 = v.pow11 + kMaxN;
    return v;
}

__device__ uint32_t mod_pow(unsigned long long base, uint32_t e) {
    unsigned long long r = 1;
    base %= kMod;
    while (e) {
        if (e & 1u) r = r * base % kMod;
        base = base * base % kMod;
        e >>= 1;
    }
    return (uint32_t)r;
}

// pow11[c] = 11^(n-1-c), pow13[r] = 13^(n-1-r); thread 0 clears the accumulators.
__global__ void k_noalloc_tables(void *scratch, uint32_t n) {
    const ScratchView s = view(scratch);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        s.acc[0] = 0;
        s.acc[1] = 0;
    }
    if (i < n) {
        s.pow11[i] = mod_pow(11, n - 1 - i);
        s.pow13[i] = mod_pow(13, n - 1 - i);
    }
}

// Thread per row word; the hash is a sum over set bits (r, c) of
// 11^(n-1-c) * 13^(n-1-r) mod p (the closed form of cfpq-cpp/Grammar.cpp:86-97).
__global__ void k_noalloc_hash(const uint64_t *__restrict__ rows, uint32_t n, uint32_t wpr, void *scratch) {
    const ScratchView s = view(scratch);
    const size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    unsigned long long h = 0, cnt = 0;
    if (x < (size_t)n * wpr) {
        const uint32_t r = (uint32_t)(x / wpr), w = (uint32_t)(x % wpr);
        uint64_t v = rows[x];
        if (w == wpr - 1 && (n & 63)) v &= (1ULL << (n & 63)) - 1;  // columns >= n are not part of the matrix
        if (v) {
            cnt = __popcll(v);
            unsigned long long line = 0;
            while (v) {
                const int b = __ffsll((long long)v) - 1;
                v &= v - 1;
                line += s.pow11[64 * w + b];
            }
            h = (line % kMod) * s.pow13[r] % kMod;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        h += __shfl_down_sync(0xffffffffu, h, o);
        cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (h) atomicAdd(s.acc, h);
        if (cnt) atomicAdd(s.acc + 1, cnt);
    }
}

__global__ void k_noalloc_finish(void *scratch, unsigned long long *out) {
    const ScratchView s = view(scratch);
    out[0] = s.acc[0] % kMod;
    out[1] = s.acc[1];
}

std::mutex g_setup_mutex;

// The array's device address belongs to the CUDA context that loaded the
// module: it is looked up again whenever the current context of the device
// is another one (a caller's own driver context, or the primary context
// created anew after cudaDeviceReset), identified by its unique context id.
struct ScratchAddr {
    void *ptr;
    unsigned long long ctx_id;
};
ScratchAddr g_scratch[kMaxDevices] = {};

thread_local char g_noalloc_error[256];

int fail(int code, const char *msg, cudaError_t e = cudaSuccess) {
    if (e != cudaSuccess)
        snprintf(g_noalloc_error, sizeof(g_noalloc_error), "%s: %s", msg, cudaGetErrorString(e));
    else
        snprintf(g_noalloc_error, sizeof(g_noalloc_error), "%s", msg);
    return code;
}

// Unique id of the current CUDA context (the driver's cuCtxGetCurrent and
// cuCtxGetId, reached through the runtime's entry-point query so that the
// library needs no link-time dependency on the driver library); 0 when the
// driver does not provide it, in which case the address is looked up on
// every call.
unsigned long long current_context_id() {
    using GetCurrent = int (*)(void **);
    using GetId = int (*)(void *, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool resolved = false;
    if (!resolved) {
        void *f = nullptr, *g = nullptr;
        cudaDriverEntryPointQueryResult r1, r2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &r1) == cudaSuccess &&
            r1 == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &g, cudaEnableDefault, &r2) == cudaSuccess &&
            r2 == cudaDriverEntryPointSuccess) {
            get_current = reinterpret_cast<GetCurrent>(f);
            get_id = reinterpret_cast<GetId>(g);
        }
        resolved = true;
    }
    void *c = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&c) != 0 || !c || get_id(c, &id) != 0) return 0;
    return id;
}

// Device address of the scratch array on `device` (which must be current).
// Looked up with cudaGetSymbolAddress at set-up, once per device and context;
// host code never uses the array's name as a device address.
int scratch_for(int device, void **out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    // 0 before the runtime made any context current: looked up again next call
    const unsigned long long id = current_context_id();
    ScratchAddr &sa = g_scratch[device];
    if (!sa.ptr || id == 0 || sa.ctx_id != id) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return fail(CFPQ_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch)", e);
        sa.ptr = p;
        sa.ctx_id = id;
    }
    *out = sa.ptr;
    return CFPQ_OK;
}

}  // namespace

extern "C" const char *cfpq_noalloc_last_error(void) { return g_noalloc_error; }

extern "C" int cfpq_hash_count_rows_noalloc(int device, const uint64_t *d_rows, uint32_t n,
                                            unsigned long long *d_out, void *stream) {
    g_noalloc_error[0] = '\0';
    if (!d_out || (n && !d_rows)) return fail(CFPQ_ERR_INVALID, "null argument");
    if (device < 0 || device >= kMaxDevices) return fail(CFPQ_ERR_INVALID, "device index out of range");
    if (n > kMaxN)
        return fail(CFPQ_ERR_UNSUPPORTED,
                    "n exceeds CFPQ_NOALLOC_MAX_N (65536); use cfpq_matrix_hash_count for larger matrices");
    int prev = -1;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return fail(CFPQ_ERR_CUDA, "cudaGetDevice", e);
    if (prev != device && (e = cudaSetDevice(device)) != cudaSuccess) return fail(CFPQ_ERR_CUDA, "cudaSetDevice", e);
    void *scratch = nullptr;
    int rc = scratch_for(device, &scratch);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (rc == CFPQ_OK) {
        const uint32_t wpr = (n + 63) / 64;
        const size_t words = (size_t)n * wpr;
        k_noalloc_tables<<<(n + 255) / 256 ? (n + 255) / 256 : 1, 256, 0, s>>>(scratch, n);
        if (words) k_noalloc_hash<<<(unsigned)((words + 255) / 256), 256, 0, s>>>(d_rows, n, wpr, scratch);
        k_noalloc_finish<<<1, 1, 0, s>>>(scratch, d_out);
        e = cudaGetLastError();
        if (e != cudaSuccess) rc = fail(CFPQ_ERR_CUDA, "kernel launch", e);
    }
    if (prev != device && prev >= 0) cudaSetDevice(prev);
    return rc;
}
