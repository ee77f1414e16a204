// hase_proposal.cu -- the learned importance proposal of libhase_b200.so:
// a 12 -> 64 -> 64 -> 64 -> 1 SiLU MLP on the sm_100a tensor cores.
//
// One CTA of 128 threads runs tiles of 128 rows (row = one (sample, slice,
// prism) pair, thread t owns row t).  Per tile:
//   features (bf16) -> smem A0 [128 x 16]
//   tcgen05.mma  A0 x W1^T -> TMEM D [128 lanes x 64 columns, f32]
//   tcgen05.ld D, + b1, SiLU, bf16 -> smem A1 [128 x 64]
//   4 x tcgen05.mma (K = 16 each) A1 x W2^T -> D;  + b2, SiLU -> A2
//   4 x tcgen05.mma A2 x W3^T -> D;  + b3, SiLU -> h3 (f32 registers)
//   logit = b4 + h3 . w4 on the CUDA cores.
// Operands live in shared memory in the canonical no-swizzle K-major layout
// of the tensor-core descriptors: 8-row x 16-byte core matrices, element
// (r, k) of a [rows x K] bf16 matrix at
//   (r / 8) * (K * 16) + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
// i.e. leading-dimension offset 128 B (next 8 k), stride offset K * 16 B
// (next 8 rows).  One thread issues the MMAs and commits them to an mbarrier;
// every wait on it is bounded (error flag + clean TMEM release on timeout).
#include "hase_b200_proposal.h"
#include "hase_host.cuh"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

using namespace hase;

namespace {

constexpr int kFeat = HASE_PROPOSAL_FEATURES;
constexpr int kHid = HASE_PROPOSAL_HIDDEN;
constexpr int kIn = 16;     // padded input width: one K = 16 MMA
constexpr int kTile = 128;  // rows per tile (MMA M)
constexpr uint32_t kSpinLimit = 1u << 22;  // mbarrier polls before the kernel gives up

// parameter offsets in the FP32 master vector
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kFeat * kHid;
constexpr int kOffW2 = kOffB1 + kHid;
constexpr int kOffB2 = kOffW2 + kHid * kHid;
constexpr int kOffW3 = kOffB2 + kHid;
constexpr int kOffB3 = kOffW3 + kHid * kHid;
constexpr int kOffW4 = kOffB3 + kHid;
constexpr int kOffB4 = kOffW4 + kHid;
static_assert(kOffB4 + 1 == HASE_PROPOSAL_PARAMS, "parameter layout");

// shared-memory images (bytes)
constexpr uint32_t kW1Bytes = kHid * kIn * 2;    // [64 n][16 k]
constexpr uint32_t kW2Bytes = kHid * kHid * 2;   // [64 n][64 k]
constexpr uint32_t kWBlobBytes = kW1Bytes + 2 * kW2Bytes;
constexpr uint32_t kA0Bytes = kTile * kIn * 2;
constexpr uint32_t kA1Bytes = kTile * kHid * 2;
constexpr int kVecFloats = 4 * kHid + 1;          // b1 b2 b3 w4 b4

struct SmemMap {
    static constexpr uint32_t w1 = 0;
    static constexpr uint32_t w2 = w1 + kW1Bytes;
    static constexpr uint32_t w3 = w2 + kW2Bytes;
    static constexpr uint32_t a0 = w3 + kW2Bytes;
    static constexpr uint32_t a1 = a0 + kA0Bytes;
    static constexpr uint32_t a2 = a1 + kA1Bytes;
    static constexpr uint32_t vec = a2 + kA1Bytes;
    static constexpr uint32_t bar = (vec + kVecFloats * 4 + 15) & ~15u;
    static constexpr uint32_t tslot = bar + 8;
    static constexpr uint32_t bytes = tslot + 8;
};
constexpr uint32_t kSmemBytes = SmemMap::bytes + 1024;  // + alignment slack

__host__ __device__ constexpr uint32_t canonOffset(uint32_t r, uint32_t k, uint32_t K) {
    return (r >> 3) * (K * 16u) + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// ----------------------------------------------------------- tcgen05 ----
__device__ __forceinline__ uint32_t smemU32(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

// Shared-memory matrix descriptor: no swizzle, offsets in 16-byte units,
// descriptor version 1 (bits 46-47) as the sm_100 tensor cores expect.
__device__ __forceinline__ uint64_t smemDesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: D f32 (bits 4-5 = 1), A and B bf16
// (bits 7-9 and 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t kIdescM128N64 = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mmaBf16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(kIdescM128N64), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mmaCommit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ bool mbarWait(uint32_t bar, uint32_t parity) {
    for (uint32_t it = 0; it < kSpinLimit; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void fenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 columns of this thread's TMEM lane; the wait for the load is part of the
// same statement, so no use of the registers can be scheduled before it.
__device__ __forceinline__ void tmemLd16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ float silu(float v) { return v / (1.0f + __expf(-v)); }

__device__ __forceinline__ uint32_t packBf16(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// Shared state of one CTA.
struct Tile {
    uint8_t* base;      // 1024-aligned generic pointer to the smem map
    uint32_t sbase;     // its shared-window address
    uint32_t tmem;      // TMEM accumulator (lane 0, first column)
    uint32_t parity;    // next mbarrier phase to wait for
    bool ok;            // false after a timed-out wait
};

// Reads this thread's row of the accumulator (64 f32 columns).
__device__ __forceinline__ void loadRow(const Tile& T, float (&acc)[kHid]) {
    const uint32_t lane0 = (threadIdx.x & ~31u) << 16;
#pragma unroll
    for (int q = 0; q < kHid / 16; ++q) {
        uint32_t r[16];
        tmemLd16(T.tmem + lane0 + uint32_t(16 * q), r);
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[16 * q + j] = __uint_as_float(r[j]);
    }
}

// Issues the MMAs of one layer (K = kIn or kHid) from thread 0 and waits for them.
__device__ __forceinline__ void runLayer(Tile& T, uint32_t aOff, uint32_t wOff, uint32_t K) {
    if (threadIdx.x == 0) {
        fenceAfterSync();
        const uint32_t sbo = K * 16u;
        for (uint32_t kk = 0; kk < K / 16u; ++kk) {
            const uint64_t a = smemDesc(T.sbase + aOff + kk * 256u, 128u, sbo);
            const uint64_t b = smemDesc(T.sbase + wOff + kk * 256u, 128u, sbo);
            mmaBf16(T.tmem, a, b, kk > 0 ? 1u : 0u);
        }
        mmaCommit(T.sbase + SmemMap::bar);
    }
    if (!mbarWait(T.sbase + SmemMap::bar, T.parity)) T.ok = false;
    T.parity ^= 1u;
    fenceAfterSync();
}

// Bias + SiLU of the accumulator row, stored as bf16 row `threadIdx.x` of the
// next layer's A operand (K = 64).
__device__ __forceinline__ void epilogueToSmem(Tile& T, const float* bias, uint32_t outOff) {
    float acc[kHid];
    loadRow(T, acc);
    const uint32_t t = threadIdx.x;
    uint8_t* out = T.base + outOff + (t >> 3) * (kHid * 16u) + (t & 7u) * 16u;
#pragma unroll
    for (int c = 0; c < kHid / 8; ++c) {
        uint4 v;
        v.x = packBf16(silu(acc[8 * c + 0] + bias[8 * c + 0]), silu(acc[8 * c + 1] + bias[8 * c + 1]));
        v.y = packBf16(silu(acc[8 * c + 2] + bias[8 * c + 2]), silu(acc[8 * c + 3] + bias[8 * c + 3]));
        v.z = packBf16(silu(acc[8 * c + 4] + bias[8 * c + 4]), silu(acc[8 * c + 5] + bias[8 * c + 5]));
        v.w = packBf16(silu(acc[8 * c + 6] + bias[8 * c + 6]), silu(acc[8 * c + 7] + bias[8 * c + 7]));
        *reinterpret_cast<uint4*>(out + c * 128u) = v;
    }
    fenceBeforeSync();
    fenceProxyAsync();
    __syncthreads();
}

// Writes this thread's feature row (kFeat floats, padded to 16) into A0.
__device__ __forceinline__ void storeFeatures(Tile& T, const float (&f)[kFeat]) {
    const uint32_t t = threadIdx.x;
    uint8_t* out = T.base + SmemMap::a0 + (t >> 3) * (kIn * 16u) + (t & 7u) * 16u;
    uint4 v0, v1;
    v0.x = packBf16(f[0], f[1]);
    v0.y = packBf16(f[2], f[3]);
    v0.z = packBf16(f[4], f[5]);
    v0.w = packBf16(f[6], f[7]);
    v1.x = packBf16(f[8], f[9]);
    v1.y = packBf16(f[10], f[11]);
    v1.z = 0u;
    v1.w = 0u;
    *reinterpret_cast<uint4*>(out) = v0;
    *reinterpret_cast<uint4*>(out + 128u) = v1;
    fenceProxyAsync();
    __syncthreads();
}

// The three tensor-core layers and the output layer for the rows in A0.
__device__ __forceinline__ float mlpTile(Tile& T) {
    const float* vec = reinterpret_cast<const float*>(T.base + SmemMap::vec);
    runLayer(T, SmemMap::a0, SmemMap::w1, kIn);
    epilogueToSmem(T, vec, SmemMap::a1);
    runLayer(T, SmemMap::a1, SmemMap::w2, kHid);
    epilogueToSmem(T, vec + kHid, SmemMap::a2);
    runLayer(T, SmemMap::a2, SmemMap::w3, kHid);
    float acc[kHid];
    loadRow(T, acc);
    const float* b3 = vec + 2 * kHid;
    const float* w4 = vec + 3 * kHid;
    float logit = vec[4 * kHid];
#pragma unroll
    for (int n = 0; n < kHid; ++n) logit = fmaf(silu(acc[n] + b3[n]), w4[n], logit);
    fenceBeforeSync();
    __syncthreads();  // TMEM reads done before the next tile's MMA overwrites D
    return logit;
}

// CTA prologue: smem map, weight images, TMEM and the mbarrier.
__device__ __forceinline__ bool tileBegin(Tile& T, uint8_t* dyn, const uint4* wimg, const float* vec) {
    const uint32_t raw = smemU32(dyn);
    const uint32_t pad = (1024u - (raw & 1023u)) & 1023u;
    T.base = dyn + pad;
    T.sbase = raw + pad;
    T.parity = 0;
    T.ok = true;
    uint4* w = reinterpret_cast<uint4*>(T.base + SmemMap::w1);
    for (uint32_t k = threadIdx.x; k < kWBlobBytes / 16u; k += blockDim.x) w[k] = wimg[k];
    float* v = reinterpret_cast<float*>(T.base + SmemMap::vec);
    for (uint32_t k = threadIdx.x; k < uint32_t(kVecFloats); k += blockDim.x) v[k] = vec[k];
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(T.sbase + SmemMap::tslot),
                     "r"(uint32_t(kHid)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(T.sbase + SmemMap::bar), "r"(1u));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fenceProxyAsync();
    fenceBeforeSync();
    __syncthreads();
    fenceAfterSync();
    T.tmem = *reinterpret_cast<volatile uint32_t*>(T.base + SmemMap::tslot);
    return true;
}

__device__ __forceinline__ void tileEnd(Tile& T, int* error) {
    fenceBeforeSync();
    __syncthreads();
    if (threadIdx.x < 32) {
        fenceAfterSync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(T.tmem), "r"(uint32_t(kHid)));
    }
    if (!T.ok && threadIdx.x == 0) atomicExch(error, 1);
}

// ---------------------------------------------------- explicit features ----
struct ForwardLaunch {
    const uint4* wimg;
    const float* vec;
    const float* features;  // [rows][kFeat]
    float* logits;          // [rows]
    uint32_t rows;
    int* error;
};

__global__ void __launch_bounds__(kTile, 1) mlpForwardKernel(const ForwardLaunch P) {
    extern __shared__ uint8_t dynSmem[];
    Tile T;
    tileBegin(T, dynSmem, P.wimg, P.vec);
    const uint32_t tiles = (P.rows + kTile - 1) / kTile;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t row = tile * kTile + threadIdx.x;
        float f[kFeat];
#pragma unroll
        for (int j = 0; j < kFeat; ++j) f[j] = row < P.rows ? P.features[size_t(row) * kFeat + j] : 0.0f;
        storeFeatures(T, f);
        const float logit = mlpTile(T);
        if (row < P.rows) P.logits[row] = logit;
        if (!__syncthreads_and(T.ok)) break;
    }
    tileEnd(T, P.error);
}

}  // namespace

// ------------------------------------------------------------ host side ----
namespace {

uint16_t bf16Bits(float x) {  // round to nearest even
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7F800000u) == 0x7F800000u) return uint16_t(u >> 16);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return uint16_t(u >> 16);
}

float bf16Round(float x) {
    const uint32_t u = uint32_t(bf16Bits(x)) << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// smem images of W1^T, W2^T, W3^T ([out][in], bf16, canonical K-major) and
// the FP32 vector b1 b2 b3 w4 (bf16-rounded) b4.
void packImages(const std::vector<float>& p, std::vector<uint8_t>& img, std::vector<float>& vec) {
    img.assign(kWBlobBytes, 0);
    auto put = [&](uint32_t base, uint32_t n, uint32_t k, uint32_t K, float v) {
        const uint16_t b = bf16Bits(v);
        std::memcpy(&img[base + canonOffset(n, k, K)], &b, 2);
    };
    for (uint32_t n = 0; n < uint32_t(kHid); ++n) {
        for (uint32_t k = 0; k < uint32_t(kFeat); ++k) put(SmemMap::w1, n, k, kIn, p[kOffW1 + k * kHid + n]);
        for (uint32_t k = 0; k < uint32_t(kHid); ++k) {
            put(SmemMap::w2, n, k, kHid, p[kOffW2 + k * kHid + n]);
            put(SmemMap::w3, n, k, kHid, p[kOffW3 + k * kHid + n]);
        }
    }
    vec.assign(kVecFloats, 0.0f);
    for (int n = 0; n < kHid; ++n) {
        vec[n] = p[kOffB1 + n];
        vec[kHid + n] = p[kOffB2 + n];
        vec[2 * kHid + n] = p[kOffB3 + n];
        vec[3 * kHid + n] = bf16Round(p[kOffW4 + n]);
    }
    vec[4 * kHid] = p[kOffB4];
}

}  // namespace

struct hase_proposal {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t numSMs = 0;
    std::vector<float> params;
    DevBuf<uint4> wimg;
    DevBuf<float> vec;
    DevBuf<int> error;
};

namespace {

hase_status uploadParams(hase_proposal* net) {
    std::vector<uint8_t> img;
    std::vector<float> vec;
    packImages(net->params, img, vec);
    HASE_CUDA(net->wimg.ensure(kWBlobBytes / 16));
    HASE_CUDA(net->vec.ensure(kVecFloats));
    HASE_CUDA(cudaMemcpyAsync(net->wimg.p, img.data(), kWBlobBytes, cudaMemcpyHostToDevice, net->stream));
    HASE_CUDA(cudaMemcpyAsync(net->vec.p, vec.data(), kVecFloats * sizeof(float), cudaMemcpyHostToDevice, net->stream));
    HASE_CUDA(cudaStreamSynchronize(net->stream));
    return HASE_OK;
}

uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

hase_status checkError(hase_proposal* net) {
    int err = 0;
    HASE_CUDA(cudaMemcpyAsync(&err, net->error.p, sizeof(int), cudaMemcpyDeviceToHost, net->stream));
    HASE_CUDA(cudaStreamSynchronize(net->stream));
    if (err) return fail(HASE_DEVICE_TIMEOUT, "a tensor-core wait of the proposal network timed out");
    return HASE_OK;
}

}  // namespace

extern "C" {

hase_status hase_proposal_create(int device, uint32_t seed, hase_proposal** out) {
    if (!out) return fail(HASE_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(HASE_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= count) return fail(HASE_INVALID_ARGUMENT, "device %d out of range", device);
    hase_proposal* net = new (std::nothrow) hase_proposal();
    if (!net) return fail(HASE_OUT_OF_MEMORY, "host allocation failed");
    net->device = device;
    // uniform fan-in initialisation U(-1/sqrt(fan_in), 1/sqrt(fan_in)), zero biases
    net->params.assign(HASE_PROPOSAL_PARAMS, 0.0f);
    uint64_t s = 0x5DEECE66Dull ^ (uint64_t(seed) << 20);
    auto uni = [&](float bound) { return float((double(splitmix(s) >> 11) * 0x1.0p-53 * 2.0 - 1.0) * bound); };
    for (int i = 0; i < kFeat * kHid; ++i) net->params[kOffW1 + i] = uni(1.0f / std::sqrt(float(kFeat)));
    for (int i = 0; i < kHid * kHid; ++i) net->params[kOffW2 + i] = uni(1.0f / std::sqrt(float(kHid)));
    for (int i = 0; i < kHid * kHid; ++i) net->params[kOffW3 + i] = uni(1.0f / std::sqrt(float(kHid)));
    for (int i = 0; i < kHid; ++i) net->params[kOffW4 + i] = uni(1.0f / std::sqrt(float(kHid)));
    auto cleanup = [&](hase_status st) {
        hase_proposal_destroy(net);
        return st;
    };
    if (cudaSetDevice(device) != cudaSuccess) return cleanup(fail(HASE_CUDA_ERROR, "cudaSetDevice failed"));
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return cleanup(fail(HASE_CUDA_ERROR, "cannot query the SM count"));
    net->numSMs = uint32_t(sms);
    if (cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking) != cudaSuccess)
        return cleanup(fail(HASE_CUDA_ERROR, "stream creation failed"));
    if (net->error.ensure(1) != cudaSuccess) return cleanup(fail(HASE_OUT_OF_MEMORY, "device allocation failed"));
    if (cudaMemset(net->error.p, 0, sizeof(int)) != cudaSuccess)
        return cleanup(fail(HASE_CUDA_ERROR, "cudaMemset failed"));
    const hase_status st = uploadParams(net);
    if (st != HASE_OK) return cleanup(st);
    *out = net;
    return HASE_OK;
}

hase_status hase_proposal_destroy(hase_proposal* net) {
    if (!net) return HASE_OK;
    cudaSetDevice(net->device);
    if (net->stream) {
        cudaStreamSynchronize(net->stream);
        cudaStreamDestroy(net->stream);
    }
    delete net;
    return HASE_OK;
}

hase_status hase_proposal_get_params(hase_proposal* net, float* params) {
    if (!net || !params) return fail(HASE_INVALID_ARGUMENT, "null argument");
    std::memcpy(params, net->params.data(), sizeof(float) * HASE_PROPOSAL_PARAMS);
    return HASE_OK;
}

hase_status hase_proposal_set_params(hase_proposal* net, const float* params) {
    if (!net || !params) return fail(HASE_INVALID_ARGUMENT, "null argument");
    for (int i = 0; i < HASE_PROPOSAL_PARAMS; ++i)
        if (!std::isfinite(params[i])) return fail(HASE_INVALID_ARGUMENT, "parameter %d is not finite", i);
    net->params.assign(params, params + HASE_PROPOSAL_PARAMS);
    HASE_CUDA(cudaSetDevice(net->device));
    return uploadParams(net);
}

hase_status hase_proposal_forward(hase_proposal* net, uint32_t rows, const float* features, float* logits) {
    if (!net || (rows && (!features || !logits))) return fail(HASE_INVALID_ARGUMENT, "null argument");
    if (rows == 0) return HASE_OK;
    HASE_CUDA(cudaSetDevice(net->device));
    DevBuf<float> f, l;
    HASE_CUDA(f.ensure(size_t(rows) * kFeat));
    HASE_CUDA(l.ensure(rows));
    HASE_CUDA(cudaMemcpyAsync(f.p, features, size_t(rows) * kFeat * sizeof(float), cudaMemcpyHostToDevice,
                              net->stream));
    HASE_CUDA(cudaFuncSetAttribute(mlpForwardKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemBytes)));
    const uint32_t tiles = (rows + kTile - 1) / kTile;
    const uint32_t grid = std::min(tiles, net->numSMs);
    ForwardLaunch P{net->wimg.p, net->vec.p, f.p, l.p, rows, net->error.p};
    mlpForwardKernel<<<grid, kTile, kSmemBytes, net->stream>>>(P);
    HASE_CUDA(cudaGetLastError());
    HASE_CUDA(cudaMemcpyAsync(logits, l.p, rows * sizeof(float), cudaMemcpyDeviceToHost, net->stream));
    HASE_CUDA(cudaStreamSynchronize(net->stream));
    return checkError(net);
}

}  // extern "C"
