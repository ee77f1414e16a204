// hase_mlp.cuh -- the learned-proposal MLP on the sm_100a tensor cores,
// shared by the translation units of libhase_b200.so that run it: the
// tcgen05 building blocks, the shared-memory maps of the inference and
// training tiles, the fused three-layer tile, and the network's host state.
//
// One CTA of 128 threads runs tiles of 128 rows (thread t owns row t):
// features (bf16) -> smem A0 [128 x 16]; tcgen05.mma A0 x W1^T -> TMEM
// [128 lanes x 64 f32 columns]; tcgen05.ld, + b1, SiLU, bf16 -> smem A1;
// 4 MMAs (K = 16 each) A1 x W2^T; -> A2; 4 MMAs A2 x W3^T; + b3, SiLU;
// logit = b4 + h3 . w4 on the CUDA cores.  Operands live in shared memory in
// the canonical no-swizzle K-major layout of the tensor-core descriptors:
// 8-row x 16-byte core matrices, element (r, k) of a [rows x K] bf16 matrix at
//   (r / 8) * (K * 16) + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
// i.e. leading-dimension offset 128 B (next 8 k), stride offset K * 16 B
// (next 8 rows).  One thread issues the MMAs and commits them to an mbarrier;
// every wait on it is bounded (error flag + clean TMEM release on timeout).
#pragma once

#include "hase_b200_proposal.h"
#include "hase_host.cuh"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <vector>

namespace {

constexpr int kFeat = HASE_PROPOSAL_FEATURES;
constexpr int kHid = HASE_PROPOSAL_HIDDEN;
constexpr int kIn = 16;     // padded input width: one K = 16 MMA
constexpr int kTile = 128;  // rows per tile (MMA M)
constexpr int kMlpBlocksPerSM = 5;  // inference CTAs per SM (shared memory ~41 KB, 64 TMEM columns, <= 102 registers)
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
constexpr uint32_t kWFwdBytes = kW1Bytes + 2 * kW2Bytes;   // W1^T W2^T W3^T (forward)
constexpr uint32_t kWBlobBytes = kWFwdBytes + 2 * kW2Bytes;  // + W2, W3 untransposed (backward)
constexpr uint32_t kA0Bytes = kTile * kIn * 2;
constexpr uint32_t kA1Bytes = kTile * kHid * 2;
constexpr int kVecFloats = 4 * kHid + 1;          // b1 b2 b3 w4 b4

// Inference: forward weight images, the feature rows and one activation buffer
// shared by the inputs of layers 2 and 3 (the layer-2 epilogue writes it only
// after the MMAs that read it have completed), 64 TMEM columns (one
// accumulator reused by the three layers).
struct SmemMap {
    static constexpr uint32_t wBytes = kWFwdBytes;
    static constexpr uint32_t tmemCols = 64;
    static constexpr uint32_t w1 = 0;
    static constexpr uint32_t w2 = w1 + kW1Bytes;
    static constexpr uint32_t w3 = w2 + kW2Bytes;
    static constexpr uint32_t a0 = w3 + kW2Bytes;
    static constexpr uint32_t a1 = a0 + kA0Bytes;
    static constexpr uint32_t a2 = a1;
    static constexpr uint32_t vec = a1 + kA1Bytes;
    static constexpr uint32_t bar = (vec + kVecFloats * 4 + 15) & ~15u;
    static constexpr uint32_t tslot = bar + 8;
    static constexpr uint32_t bytes = tslot + 8;
};
constexpr uint32_t kSmemBytes = SmemMap::bytes + 1024;  // + alignment slack

// Training: also the backward weight images (W2, W3 as [in][out]: the B
// operands of dz2 W2^T and dz3 W3^T), dz as the bf16 operand of the backward
// and weight-gradient products, silu'(z1 + b1) as bf16 rows (z1's TMEM
// columns are reused by layer 3), the warps' partial bias sums, and 256 TMEM
// columns, so two CTAs share an SM: z1, then z3 and the backward products
// (0); z2 (64); the weight gradients accumulated over all tiles of the CTA
// as M = 64 accumulators, dW3 and dW2 interleaved in one 64-column block
// (lanes 0-15 and 16-31 of each warp quarter, 128) and dW1^T (lanes 0-15,
// 192).
struct TrainSmem {
    static constexpr uint32_t wBytes = kWBlobBytes;
    static constexpr uint32_t tmemCols = 256;
    static constexpr uint32_t colGradW32 = 128;  // dW3 in lanes 0-15, dW2 in lanes 16-31
    static constexpr uint32_t colGradW1 = 192;
    static constexpr uint32_t w1 = 0;
    static constexpr uint32_t w2 = w1 + kW1Bytes;
    static constexpr uint32_t w3 = w2 + kW2Bytes;
    static constexpr uint32_t w2b = w3 + kW2Bytes;
    static constexpr uint32_t w3b = w2b + kW2Bytes;
    static constexpr uint32_t a0 = w3b + kW2Bytes;
    static constexpr uint32_t a1 = a0 + kA0Bytes;
    static constexpr uint32_t a2 = a1 + kA1Bytes;
    static constexpr uint32_t dzb = a2 + kA1Bytes;
    static constexpr uint32_t ds1 = dzb + kA1Bytes;  // silu'(z1 + b1), bf16, the canonical row layout
    static constexpr uint32_t red = ds1 + kA1Bytes;  // [4 warps][64] column partials, [4] row-sum partials
    static constexpr uint32_t vec = red + (4 * kHid + 4) * 4;
    static constexpr uint32_t bar = (vec + kVecFloats * 4 + 15) & ~15u;
    static constexpr uint32_t tslot = bar + 8;
    static constexpr uint32_t bytes = tslot + 8;
};
constexpr uint32_t kTrainSmemBytes = TrainSmem::bytes + 1024;
static_assert(2 * (kTrainSmemBytes + 1024) <= 228u * 1024u, "two training CTAs per SM");
static_assert(SmemMap::w3 == TrainSmem::w3, "the forward images lead the weight blob in both maps");

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
// The weight-gradient products: A and B MN-major (bits 15 and 16), M = 64.
constexpr uint32_t kIdescGradN64 =
    (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((64u >> 3) << 17) | ((64u >> 4) << 24);
constexpr uint32_t kIdescGradN16 =
    (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((16u >> 3) << 17) | ((64u >> 4) << 24);

__device__ __forceinline__ void mmaBf16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate,
                                        uint32_t idesc = kIdescM128N64) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
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

// SiLU with the fast reciprocal (FP32 error of a few ulp, far below the BF16
// rounding that follows); v -> -inf gives -0.
__device__ __forceinline__ float silu(float v) { return __fdividef(v, 1.0f + __expf(-v)); }

// SiLU from one special-function instruction, for the proposal inside the
// phi-ASE solve: v sigmoid(v) = h + h tanh(h), h = v / 2, with the hardware
// tanh approximation (tanh.approx.f32).  Against the exact form it differs by
// the approximation's relative error (about 2^-11), below the BF16 rounding
// that follows on the hidden layers; the solve weights every ray by the
// proposal it was actually drawn from, so the estimate stays unbiased.
__device__ __forceinline__ float siluTanh(float v) {
    const float h = 0.5f * v;
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(h));
    return fmaf(h, t, h);
}

template <bool FAST>
__device__ __forceinline__ float act(float v) {
    return FAST ? siluTanh(v) : silu(v);
}

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

// Reads this thread's row of the accumulator at TMEM column `col` (64 f32 columns).
__device__ __forceinline__ void loadRow(const Tile& T, uint32_t col, float (&acc)[kHid]) {
    const uint32_t lane0 = (threadIdx.x & ~31u) << 16;
#pragma unroll
    for (int q = 0; q < kHid / 16; ++q) {
        uint32_t r[16];
        tmemLd16(T.tmem + lane0 + col + uint32_t(16 * q), r);
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[16 * q + j] = __uint_as_float(r[j]);
    }
}

// Reads N (a multiple of 16) accumulator columns of this thread's row from
// TMEM column `col`.
template <int N>
__device__ __forceinline__ void loadCols(const Tile& T, uint32_t col, float (&acc)[N]) {
    const uint32_t lane0 = (threadIdx.x & ~31u) << 16;
#pragma unroll
    for (int q = 0; q < N / 16; ++q) {
        uint32_t r[16];
        tmemLd16(T.tmem + lane0 + col + uint32_t(16 * q), r);
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[16 * q + j] = __uint_as_float(r[j]);
    }
}

// Issues the MMAs of one product [128 x K] x [64 x K]^T (K = kIn or kHid)
// into TMEM column `col` from thread 0 and commits them to the mbarrier.
__device__ __forceinline__ void issueLayer(Tile& T, uint32_t aOff, uint32_t wOff, uint32_t K, uint32_t col,
                                           uint32_t barOff) {
    if (threadIdx.x == 0) {
        fenceAfterSync();
        const uint32_t sbo = K * 16u;
        for (uint32_t kk = 0; kk < K / 16u; ++kk) {
            const uint64_t a = smemDesc(T.sbase + aOff + kk * 256u, 128u, sbo);
            const uint64_t b = smemDesc(T.sbase + wOff + kk * 256u, 128u, sbo);
            mmaBf16(T.tmem + col, a, b, kk > 0 ? 1u : 0u);
        }
        mmaCommit(T.sbase + barOff);
    }
}

// Issues (from thread 0, without a commit) the weight-gradient product
// D[m][n] (+)= sum_r A[r][m] B[r][n] over the tile's 128 rows into TMEM
// column `col` (an M = 64 accumulator: row m in TMEM lane 32 (m / 16) +
// m % 16, the first 16 lanes of warp m / 16's lane quarter).  A ([128 x 64]) and B ([128 x bWidth])
// are row-major bf16 images in the canonical layout of the forward operands
// (8-row x 16-byte core matrices, 8-row groups width x 16 bytes apart), which
// are MN-major operands of the transposed product: SBO = 128 bytes (next 8
// columns), LBO = width x 16 bytes (next 8 rows), 16 rows per MMA.
// accumulate = false starts the accumulator with this tile.
__device__ __forceinline__ void issueGradient(const Tile& T, uint32_t aOff, uint32_t bOff, uint32_t bWidth,
                                              uint32_t col, uint32_t idesc, bool accumulate) {
    const uint32_t aRows = kHid * 16u, bRows = bWidth * 16u;
    for (uint32_t kk = 0; kk < uint32_t(kTile) / 16u; ++kk) {
        const uint64_t a = smemDesc(T.sbase + aOff + kk * 2u * aRows, aRows, 128u);
        const uint64_t b = smemDesc(T.sbase + bOff + kk * 2u * bRows, bRows, 128u);
        mmaBf16(T.tmem + col, a, b, (accumulate || kk > 0) ? 1u : 0u, idesc);
    }
}

__device__ __forceinline__ void waitLayer(Tile& T, uint32_t barOff) {
    if (!mbarWait(T.sbase + barOff, T.parity)) T.ok = false;
    T.parity ^= 1u;
    fenceAfterSync();
}

__device__ __forceinline__ void runLayer(Tile& T, uint32_t aOff, uint32_t wOff, uint32_t K, uint32_t col,
                                         uint32_t barOff) {
    issueLayer(T, aOff, wOff, K, col, barOff);
    waitLayer(T, barOff);
}

// Bias + SiLU of the accumulator row, stored as bf16 row `threadIdx.x` of the
// next layer's A operand (K = 64).
// The row is processed in two halves of 32 columns, which keeps the register
// count low enough for the inference occupancy target.
template <bool FAST = false>
__device__ __forceinline__ void epilogueToSmem(Tile& T, uint32_t col, const float* bias, uint32_t outOff) {
    const uint32_t t = threadIdx.x;
    uint8_t* out = T.base + outOff + (t >> 3) * (kHid * 16u) + (t & 7u) * 16u;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        constexpr int kHalf = kHid / 2;
        float acc[kHalf];
        loadCols<kHalf>(T, col + uint32_t(h * kHalf), acc);
        const float* b = bias + h * kHalf;
#pragma unroll
        for (int c = 0; c < kHalf / 8; ++c) {
            uint4 v;
            v.x = packBf16(act<FAST>(acc[8 * c + 0] + b[8 * c + 0]), act<FAST>(acc[8 * c + 1] + b[8 * c + 1]));
            v.y = packBf16(act<FAST>(acc[8 * c + 2] + b[8 * c + 2]), act<FAST>(acc[8 * c + 3] + b[8 * c + 3]));
            v.z = packBf16(act<FAST>(acc[8 * c + 4] + b[8 * c + 4]), act<FAST>(acc[8 * c + 5] + b[8 * c + 5]));
            v.w = packBf16(act<FAST>(acc[8 * c + 6] + b[8 * c + 6]), act<FAST>(acc[8 * c + 7] + b[8 * c + 7]));
            *reinterpret_cast<uint4*>(out + uint32_t(h * kHalf / 8 + c) * 128u) = v;
        }
    }
    fenceBeforeSync();
    fenceProxyAsync();
    __syncthreads();
}

// Writes this thread's feature row (kFeat floats, padded to 16) into A0.
__device__ __forceinline__ void storeFeatures(Tile& T, uint32_t a0Off, const float (&f)[kFeat]) {
    const uint32_t t = threadIdx.x;
    uint8_t* out = T.base + a0Off + (t >> 3) * (kIn * 16u) + (t & 7u) * 16u;
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

// The three tensor-core layers and the output layer for the rows in A0
// (FAST: the single-instruction SiLU of the in-solve proposal).
template <bool FAST = false>
__device__ __forceinline__ float mlpTile(Tile& T) {
    const float* vec = reinterpret_cast<const float*>(T.base + SmemMap::vec);
    runLayer(T, SmemMap::a0, SmemMap::w1, kIn, 0, SmemMap::bar);
    epilogueToSmem<FAST>(T, 0, vec, SmemMap::a1);
    runLayer(T, SmemMap::a1, SmemMap::w2, kHid, 0, SmemMap::bar);
    epilogueToSmem<FAST>(T, 0, vec + kHid, SmemMap::a2);
    runLayer(T, SmemMap::a2, SmemMap::w3, kHid, 0, SmemMap::bar);
    const float* b3 = vec + 2 * kHid;
    const float* w4 = vec + 3 * kHid;
    float logit = vec[4 * kHid];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        constexpr int kHalf = kHid / 2;
        float acc[kHalf];
        loadCols<kHalf>(T, uint32_t(h * kHalf), acc);
#pragma unroll
        for (int n = 0; n < kHalf; ++n)
            logit = fmaf(act<FAST>(acc[n] + b3[h * kHalf + n]), w4[h * kHalf + n], logit);
    }
    fenceBeforeSync();
    __syncthreads();  // TMEM reads done before the next tile's MMA overwrites D
    return logit;
}

// CTA prologue: smem map, weight images, TMEM and the mbarrier.
template <typename Map>
__device__ __forceinline__ bool tileBegin(Tile& T, uint8_t* dyn, const uint4* wimg, const float* vec) {
    const uint32_t raw = smemU32(dyn);
    const uint32_t pad = (1024u - (raw & 1023u)) & 1023u;
    T.base = dyn + pad;
    T.sbase = raw + pad;
    T.parity = 0;
    T.ok = true;
    uint4* w = reinterpret_cast<uint4*>(T.base + SmemMap::w1);
    for (uint32_t k = threadIdx.x; k < Map::wBytes / 16u; k += blockDim.x) w[k] = wimg[k];
    float* v = reinterpret_cast<float*>(T.base + Map::vec);
    for (uint32_t k = threadIdx.x; k < uint32_t(kVecFloats); k += blockDim.x) v[k] = vec[k];
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(T.sbase + Map::tslot),
                     "r"(Map::tmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(T.sbase + Map::bar), "r"(1u));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fenceProxyAsync();
    fenceBeforeSync();
    __syncthreads();
    fenceAfterSync();
    T.tmem = *reinterpret_cast<volatile uint32_t*>(T.base + Map::tslot);
    return true;
}

template <typename Map>
__device__ __forceinline__ void tileEnd(Tile& T, int* error) {
    fenceBeforeSync();
    __syncthreads();
    if (threadIdx.x < 32) {
        fenceAfterSync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(T.tmem), "r"(Map::tmemCols));
    }
    if (!T.ok && threadIdx.x == 0) atomicExch(error, 1);
}

}  // namespace

struct hase_proposal {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t numSMs = 0;
    std::vector<float> params;
    hase::DevBuf<uint4> wimg;  // BF16 weight images (forward, then backward)
    hase::DevBuf<float> vec;   // b1 b2 b3 w4 b4
    hase::DevBuf<int> error;   // set by a kernel whose tensor-core wait timed out
    // training state
    hase::DevBuf<float> dparams, adamM, adamV, grad, loss;
};
