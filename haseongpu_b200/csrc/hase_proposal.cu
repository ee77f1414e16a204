// hase_proposal.cu -- the learned importance proposal of libhase_b200.so
// (include/hase_b200_proposal.h): the network on explicit feature rows,
// training (fused recompute-forward/backward tiles, per-sample softmax
// statistics, Adam, BF16 repacking on the device) and the C ABI.  The tile
// machinery itself is in hase_mlp.cuh.
#include "hase_mlp.cuh"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

using namespace hase;


namespace {

// ---------------------------------------------------- explicit features ----
struct ForwardLaunch {
    const uint4* wimg;
    const float* vec;
    const float* features;  // [rows][kFeat]
    float* logits;          // [rows]
    uint32_t rows;
    int* error;
};

__global__ void __launch_bounds__(kTile, kMlpBlocksPerSM) mlpForwardKernel(const ForwardLaunch P) {
    extern __shared__ uint8_t dynSmem[];
    Tile T;
    tileBegin<SmemMap>(T, dynSmem, P.wimg, P.vec);
    const uint32_t tiles = (P.rows + kTile - 1) / kTile;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t row = tile * kTile + threadIdx.x;
        float f[kFeat];
#pragma unroll
        for (int j = 0; j < kFeat; ++j) f[j] = row < P.rows ? P.features[size_t(row) * kFeat + j] : 0.0f;
        storeFeatures(T, SmemMap::a0, f);
        const float logit = mlpTile(T);
        if (row < P.rows) P.logits[row] = logit;
        if (!__syncthreads_and(T.ok)) break;
    }
    tileEnd<SmemMap>(T, P.error);
}

}  // namespace

// ------------------------------------------------------------- training ----
namespace {

__device__ __forceinline__ float dsilu(float z) {
    const float sg = 1.0f / (1.0f + __expf(-z));
    return sg * (1.0f + z * (1.0f - sg));
}

// g[j] += sum over the tile's rows r of h[r][i0 + j] * dz[r][o] (j < 32) and
// This thread's row of 64 values as bf16 row threadIdx.x of a canonical
// K = 64 image at off (the A operand of the backward products).
__device__ __forceinline__ void storeRowBf16(const Tile& T, uint32_t off, const float (&v)[kHid]) {
    uint8_t* out = T.base + off + (threadIdx.x >> 3) * (kHid * 16u) + (threadIdx.x & 7u) * 16u;
#pragma unroll
    for (int c = 0; c < kHid / 8; ++c) {
        uint4 w;
        w.x = packBf16(v[8 * c + 0], v[8 * c + 1]);
        w.y = packBf16(v[8 * c + 2], v[8 * c + 3]);
        w.z = packBf16(v[8 * c + 4], v[8 * c + 5]);
        w.w = packBf16(v[8 * c + 6], v[8 * c + 7]);
        *reinterpret_cast<uint4*>(out + c * 128u) = w;
    }
}

// This thread's bf16 row of a canonical K = 64 image at off, as floats.
__device__ __forceinline__ void loadRowBf16(const Tile& T, uint32_t off, float (&v)[kHid]) {
    const uint8_t* in = T.base + off + (threadIdx.x >> 3) * (kHid * 16u) + (threadIdx.x & 7u) * 16u;
#pragma unroll
    for (int c = 0; c < kHid / 8; ++c) {
        const uint4 w = *reinterpret_cast<const uint4*>(in + c * 128u);
        const uint32_t x[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            v[8 * c + 2 * e] = __uint_as_float(x[e] << 16);
            v[8 * c + 2 * e + 1] = __uint_as_float(x[e] & 0xFFFF0000u);
        }
    }
}

// The layer-1 epilogue of a training tile: h1 = silu(z1 + b1) into A1 and
// silu'(z1 + b1) into the ds1 rows (bf16), so that layer 3 can reuse z1's
// TMEM columns.
__device__ __forceinline__ void epilogueLayer1Train(Tile& T, const float* b1) {
    float z[kHid], h[kHid];
    loadRow(T, 0, z);
#pragma unroll
    for (int n = 0; n < kHid; ++n) {
        const float v = z[n] + b1[n];
        h[n] = silu(v);
        z[n] = dsilu(v);
    }
    storeRowBf16(T, TrainSmem::a1, h);
    storeRowBf16(T, TrainSmem::ds1, z);
    fenceBeforeSync();
    fenceProxyAsync();
    __syncthreads();
}

// Column sums over the tile's 128 rows of the 64-wide row v each thread holds
// (its row): a warp reduce-scatter in registers (five butterfly steps; lane
// L ends with columns 2L and 2L + 1 summed over the warp's rows), then the
// four warps' partials through shared memory: thread t < 64 adds column t to
// acc.  v is consumed.  All threads; ends with a barrier.
__device__ __forceinline__ void tileColumnSums(const Tile& T, float (&v)[kHid], float& acc) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
#pragma unroll
    for (int step = 0; step < 5; ++step) {
        const int half = 32 >> step;
        const uint32_t off = 16u >> step;
        const bool upper = (lane & off) != 0u;
#pragma unroll
        for (int i = 0; i < half; ++i) {
            const float a = v[i], b = v[i + half];
            v[i] = (upper ? b : a) + __shfl_xor_sync(0xffffffffu, upper ? a : b, off);
        }
    }
    float* red = reinterpret_cast<float*>(T.base + TrainSmem::red);
    red[warp * kHid + 2 * lane] = v[0];
    red[warp * kHid + 2 * lane + 1] = v[1];
    __syncthreads();
    if (threadIdx.x < uint32_t(kHid))
        acc += (red[threadIdx.x] + red[kHid + threadIdx.x]) + (red[2 * kHid + threadIdx.x] + red[3 * kHid + threadIdx.x]);
    __syncthreads();
}

// The sum over the tile's rows of one value per thread, added to acc by thread 0.
__device__ __forceinline__ void tileRowSum(const Tile& T, float x, float& acc) {
    for (uint32_t off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
    float* red = reinterpret_cast<float*>(T.base + TrainSmem::red) + 4 * kHid;
    if ((threadIdx.x & 31u) == 0) red[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x == 0) acc += (red[0] + red[1]) + (red[2] + red[3]);
    __syncthreads();
}

// Adds this thread's row of an M = 64 weight-gradient accumulator (TMEM
// column `col`, `cols` columns; lanes 0-15 of each warp hold rows 16 warp +
// lane) to grad[base + row * rowStride + n * colStride] for n < keep.
template <int COLS>
__device__ __forceinline__ void flushGradient(const Tile& T, uint32_t col, float* grad, uint32_t rowStride,
                                              uint32_t colStride, int keep) {
    float acc[COLS];
    loadCols<COLS>(T, col, acc);
    const uint32_t lane = threadIdx.x & 31u, row = 16u * (threadIdx.x >> 5) + lane;
    if (lane < 16u)
        for (int n = 0; n < keep; ++n) atomicAdd(grad + row * rowStride + uint32_t(n) * colStride, acc[n]);
}

struct TrainLaunch {
    const uint4* wimg;      // forward + backward images
    const float* vec;
    const float* features;  // [rows][kFeat]
    const float* dl;        // [rows]: dLoss / dlogit
    uint32_t rows;
    float* grad;            // [HASE_PROPOSAL_PARAMS], accumulated
    int* error;
};

// Recomputes the forward pass of each tile and back-propagates dL/dlogit on
// the tensor cores: per layer one commit covers the backward product (dz3
// W3^T or dz2 W2^T, over the consumed layer-3 accumulator) and the
// weight-gradient product (h2^T dz3, h1^T dz2, dz1^T x: the activation and dz
// images read as MN-major operands) that accumulates in TMEM over all tiles
// of the CTA; the bias sums run on the CUDA cores meanwhile.  Two CTAs per SM
// (256 TMEM columns each, TrainSmem).  The CTA adds its gradients to `grad`
// once.
__global__ void __launch_bounds__(kTile, 2) mlpBackwardKernel(const TrainLaunch P) {
    extern __shared__ uint8_t dynSmem[];
    Tile T;
    tileBegin<TrainSmem>(T, dynSmem, P.wimg, P.vec);
    const uint32_t t = threadIdx.x, o = t & 63u, ih = t >> 6;
    const float* vec = reinterpret_cast<const float*>(T.base + TrainSmem::vec);
    const float *b1 = vec, *b2 = vec + kHid, *b3 = vec + 2 * kHid, *w4 = vec + 3 * kHid;
    float gb1 = 0.0f, gb2 = 0.0f, gb3 = 0.0f, gw4 = 0.0f, gb4 = 0.0f;
    bool accumulate = false;  // the gradient accumulators hold a tile
    const uint32_t tiles = (P.rows + kTile - 1) / kTile;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t row = tile * kTile + t;
        float f[kFeat];
#pragma unroll
        for (int j = 0; j < kFeat; ++j) f[j] = row < P.rows ? P.features[size_t(row) * kFeat + j] : 0.0f;
        const float dl = row < P.rows ? P.dl[row] : 0.0f;
        storeFeatures(T, TrainSmem::a0, f);
        runLayer(T, TrainSmem::a0, TrainSmem::w1, kIn, 0, TrainSmem::bar);
        epilogueLayer1Train(T, b1);
        runLayer(T, TrainSmem::a1, TrainSmem::w2, kHid, 64, TrainSmem::bar);
        epilogueToSmem(T, 64, b2, TrainSmem::a2);
        runLayer(T, TrainSmem::a2, TrainSmem::w3, kHid, 0, TrainSmem::bar);  // z3 over z1
        // output layer: g_w4 = sum_r h3 dl, g_b4 = sum_r dl
        float dz[kHid];
        {
            float z[kHid];
            loadRow(T, 0, z);
#pragma unroll
            for (int n = 0; n < kHid; ++n) dz[n] = silu(z[n] + b3[n]) * dl;
        }
        tileColumnSums(T, dz, gw4);
        tileRowSum(T, dl, gb4);
        // dz3 = dl w4 * silu'(z3)
        {
            float z[kHid];
            loadRow(T, 0, z);
#pragma unroll
            for (int n = 0; n < kHid; ++n) dz[n] = dl * w4[n] * dsilu(z[n] + b3[n]);
            storeRowBf16(T, TrainSmem::dzb, dz);
        }
        fenceBeforeSync();
        fenceProxyAsync();
        __syncthreads();
        // dh2 = dz3 W3^T (over z3, read by every thread before the barrier above)
        // and g_W3 += h2^T dz3 on the tensor cores, g_b3 on the CUDA cores
        if (t == 0) {
            fenceAfterSync();
            for (uint32_t kk = 0; kk < uint32_t(kHid) / 16u; ++kk)
                mmaBf16(T.tmem, smemDesc(T.sbase + TrainSmem::dzb + kk * 256u, 128u, kHid * 16u),
                        smemDesc(T.sbase + TrainSmem::w3b + kk * 256u, 128u, kHid * 16u), kk > 0 ? 1u : 0u);
            issueGradient(T, TrainSmem::a2, TrainSmem::dzb, kHid, TrainSmem::colGradW32, kIdescGradN64, accumulate);
            mmaCommit(T.sbase + TrainSmem::bar);
        }
        tileColumnSums(T, dz, gb3);
        waitLayer(T, TrainSmem::bar);
        loadRow(T, 0, dz);
        {
            float z[kHid];
            loadRow(T, 64, z);
#pragma unroll
            for (int n = 0; n < kHid; ++n) dz[n] *= dsilu(z[n] + b2[n]);
        }
        fenceBeforeSync();
        __syncthreads();  // TMEM columns 0 (dh2) and 64 (z2) read by every warp
        storeRowBf16(T, TrainSmem::dzb, dz);
        fenceBeforeSync();
        fenceProxyAsync();
        __syncthreads();
        // dh1 = dz2 W2^T (over dh2) and g_W2 += h1^T dz2 (the lanes 16-31 half
        // of the gradient block), g_b2 meanwhile
        if (t == 0) {
            fenceAfterSync();
            for (uint32_t kk = 0; kk < uint32_t(kHid) / 16u; ++kk)
                mmaBf16(T.tmem, smemDesc(T.sbase + TrainSmem::dzb + kk * 256u, 128u, kHid * 16u),
                        smemDesc(T.sbase + TrainSmem::w2b + kk * 256u, 128u, kHid * 16u), kk > 0 ? 1u : 0u);
            issueGradient(T, TrainSmem::a1, TrainSmem::dzb, kHid, (16u << 16) + TrainSmem::colGradW32, kIdescGradN64,
                          accumulate);
            mmaCommit(T.sbase + TrainSmem::bar);
        }
        tileColumnSums(T, dz, gb2);
        waitLayer(T, TrainSmem::bar);
        loadRow(T, 0, dz);
        {
            float d1[kHid];
            loadRowBf16(T, TrainSmem::ds1, d1);
#pragma unroll
            for (int n = 0; n < kHid; ++n) dz[n] *= d1[n];
        }
        fenceBeforeSync();
        __syncthreads();  // TMEM column 0 read by every warp
        storeRowBf16(T, TrainSmem::dzb, dz);
        fenceBeforeSync();
        fenceProxyAsync();
        __syncthreads();
        // g_W1^T += dz1^T x (the bf16 features in A0, 16 columns), g_b1 meanwhile;
        // the wait keeps A0 and the dz image until the products have read them
        if (t == 0) {
            fenceAfterSync();
            issueGradient(T, TrainSmem::dzb, TrainSmem::a0, kIn, TrainSmem::colGradW1, kIdescGradN16, accumulate);
            mmaCommit(T.sbase + TrainSmem::bar);
        }
        tileColumnSums(T, dz, gb1);
        waitLayer(T, TrainSmem::bar);
        accumulate = true;
        fenceBeforeSync();
        if (!__syncthreads_and(T.ok)) break;
    }
    if (accumulate) {
        // g_W3 (lanes 0-15) and g_W2 (lanes 16-31) as [in][out] rows (row =
        // input) from the interleaved block; g_W1^T as [out][in] rows
        {
            float acc[kHid];
            loadCols<kHid>(T, TrainSmem::colGradW32, acc);
            const uint32_t lane = t & 31u, r = 16u * (t >> 5) + (lane & 15u);
            float* g = P.grad + (lane < 16u ? kOffW3 : kOffW2) + r * kHid;
            for (int n = 0; n < kHid; ++n) atomicAdd(g + n, acc[n]);
        }
        flushGradient<kIn>(T, TrainSmem::colGradW1, P.grad + kOffW1, 1u, kHid, kFeat);
    }
    if (ih == 0) {
        atomicAdd(P.grad + kOffB1 + o, gb1);
        atomicAdd(P.grad + kOffB2 + o, gb2);
        atomicAdd(P.grad + kOffB3 + o, gb3);
        atomicAdd(P.grad + kOffW4 + o, gw4);
    }
    if (t == 0) atomicAdd(P.grad + kOffB4, gb4);
    tileEnd<TrainSmem>(T, P.error);
}

// Softmax statistics of group g (rows off[g] .. off[g+1] of the step, minus
// rowBase): lse, and dl_r = w_g / G (exp(l_r - lse) - t_r / sum t); the group's
// cross entropy w_g (lse - sum t l / sum t) / G is added to *loss.
struct StatsLaunch {
    const float* logits;
    const float* targets;
    const float* groupWeights;  // or null
    const uint32_t* offsets;
    uint32_t g0, rowBase;
    float invGroups;
    float* dl;
    float* loss;
};

__device__ __forceinline__ float blockReduce(float v, float* red, bool isMax) {
    for (int o = 16; o > 0; o >>= 1) {
        const float w = __shfl_xor_sync(0xffffffffu, v, o);
        v = isMax ? fmaxf(v, w) : v + w;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    v = red[0];
    for (int k = 1; k < int(blockDim.x >> 5); ++k) v = isMax ? fmaxf(v, red[k]) : v + red[k];
    return v;
}

__global__ void __launch_bounds__(256) groupStatsKernel(const StatsLaunch S) {
    __shared__ float red[8];
    const uint32_t g = S.g0 + blockIdx.x;
    const uint32_t a = S.offsets[g] - S.rowBase, b = S.offsets[g + 1] - S.rowBase;
    float m = -INFINITY;
    for (uint32_t r = a + threadIdx.x; r < b; r += blockDim.x) m = fmaxf(m, S.logits[r]);
    m = blockReduce(m, red, true);
    float se = 0.0f, st = 0.0f, stl = 0.0f;
    for (uint32_t r = a + threadIdx.x; r < b; r += blockDim.x) {
        const float l = S.logits[r], tt = S.targets[r];
        se += __expf(l - m);
        st += tt;
        stl += tt * (l - m);
    }
    se = blockReduce(se, red, false);
    st = blockReduce(st, red, false);
    stl = blockReduce(stl, red, false);
    const float w = (S.groupWeights ? S.groupWeights[g] : 1.0f) * S.invGroups;
    const float lse = logf(se);  // relative to m
    for (uint32_t r = a + threadIdx.x; r < b; r += blockDim.x)
        S.dl[r] = st > 0.0f ? w * (__expf(S.logits[r] - m - lse) - S.targets[r] / st) : 0.0f;
    if (threadIdx.x == 0 && st > 0.0f) atomicAdd(S.loss, w * (lse - stl / st));
}

__global__ void adamKernel(float* p, float* m, float* v, const float* g, int n, float lr, float b1, float b2,
                           float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// BF16 weight images and the f32 vector from the f32 master parameters
// (the device copy of packImages).
__global__ void packKernel(const float* p, uint8_t* img, float* vec) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    constexpr uint32_t n1 = kHid * kIn, n2 = kHid * kHid;
    auto put = [&](uint32_t base, uint32_t n, uint32_t k, uint32_t K, float val) {
        *reinterpret_cast<__nv_bfloat16*>(img + base + canonOffset(n, k, K)) = __float2bfloat16_rn(val);
    };
    if (i < n1) {
        const uint32_t n = i / kIn, k = i % kIn;
        put(TrainSmem::w1, n, k, kIn, k < uint32_t(kFeat) ? p[kOffW1 + k * kHid + n] : 0.0f);
    } else if (i < n1 + 4 * n2) {
        const uint32_t j = i - n1, which = j / n2, n = (j % n2) / kHid, k = j % kHid;
        if (which == 0) put(TrainSmem::w2, n, k, kHid, p[kOffW2 + k * kHid + n]);
        else if (which == 1) put(TrainSmem::w3, n, k, kHid, p[kOffW3 + k * kHid + n]);
        else if (which == 2) put(TrainSmem::w2b, n, k, kHid, p[kOffW2 + n * kHid + k]);
        else put(TrainSmem::w3b, n, k, kHid, p[kOffW3 + n * kHid + k]);
    } else if (i < n1 + 4 * n2 + uint32_t(kVecFloats)) {
        const uint32_t j = i - n1 - 4 * n2;
        float val;
        if (j < uint32_t(kHid)) val = p[kOffB1 + j];
        else if (j < 2u * kHid) val = p[kOffB2 + j - kHid];
        else if (j < 3u * kHid) val = p[kOffB3 + j - 2 * kHid];
        else if (j < 4u * kHid) val = __bfloat162float(__float2bfloat16_rn(p[kOffW4 + j - 3 * kHid]));
        else val = p[kOffB4];
        vec[j] = val;
    }
}
constexpr uint32_t kPackThreads = kHid * kIn + 4 * kHid * kHid + kVecFloats;

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
            put(TrainSmem::w2b, n, k, kHid, p[kOffW2 + n * kHid + k]);
            put(TrainSmem::w3b, n, k, kHid, p[kOffW3 + n * kHid + k]);
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
    const uint32_t grid = std::min(tiles, net->numSMs * kMlpBlocksPerSM);
    ForwardLaunch P{net->wimg.p, net->vec.p, f.p, l.p, rows, net->error.p};
    mlpForwardKernel<<<grid, kTile, kSmemBytes, net->stream>>>(P);
    HASE_CUDA(cudaGetLastError());
    HASE_CUDA(cudaMemcpyAsync(logits, l.p, rows * sizeof(float), cudaMemcpyDeviceToHost, net->stream));
    HASE_CUDA(cudaStreamSynchronize(net->stream));
    return checkError(net);
}

}  // extern "C"

namespace {

struct DeviceBatch {
    uint32_t groups = 0, rows = 0;
    std::vector<uint32_t> offsets;
    DevBuf<uint32_t> doffsets;
    DevBuf<float> features, targets, weights, logits, dl;
    bool hasWeights = false;
};

hase_status uploadBatch(hase_proposal* net, const hase_proposal_batch* b, DeviceBatch& d) {
    if (!b || !b->offsets || b->groups == 0) return fail(HASE_INVALID_ARGUMENT, "empty training batch");
    if (b->offsets[0] != 0) return fail(HASE_INVALID_ARGUMENT, "offsets[0] must be 0");
    for (uint32_t g = 0; g < b->groups; ++g)
        if (b->offsets[g + 1] < b->offsets[g]) return fail(HASE_INVALID_ARGUMENT, "offsets must not decrease");
    d.groups = b->groups;
    d.rows = b->offsets[b->groups];
    if (d.rows == 0) return fail(HASE_INVALID_ARGUMENT, "the batch has no rows");
    if (!b->features || !b->targets) return fail(HASE_INVALID_ARGUMENT, "features and targets are required");
    for (uint32_t r = 0; r < d.rows; ++r)
        if (!(b->targets[r] >= 0.0f) || !std::isfinite(b->targets[r]))
            return fail(HASE_INVALID_ARGUMENT, "targets must be finite and >= 0");
    d.offsets.assign(b->offsets, b->offsets + b->groups + 1);
    d.hasWeights = b->groupWeights != nullptr;
    HASE_CUDA(d.doffsets.ensure(b->groups + 1));
    HASE_CUDA(d.features.ensure(size_t(d.rows) * kFeat));
    HASE_CUDA(d.targets.ensure(d.rows));
    HASE_CUDA(d.logits.ensure(d.rows));
    HASE_CUDA(d.dl.ensure(d.rows));
    HASE_CUDA(cudaMemcpyAsync(d.doffsets.p, b->offsets, (b->groups + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice,
                              net->stream));
    HASE_CUDA(cudaMemcpyAsync(d.features.p, b->features, size_t(d.rows) * kFeat * sizeof(float),
                              cudaMemcpyHostToDevice, net->stream));
    HASE_CUDA(cudaMemcpyAsync(d.targets.p, b->targets, d.rows * sizeof(float), cudaMemcpyHostToDevice, net->stream));
    if (d.hasWeights) {
        HASE_CUDA(d.weights.ensure(b->groups));
        HASE_CUDA(cudaMemcpyAsync(d.weights.p, b->groupWeights, b->groups * sizeof(float), cudaMemcpyHostToDevice,
                                  net->stream));
    }
    return HASE_OK;
}

// Loss (added to *dLoss) and gradient (added to dGrad) of groups [g0, g1).
hase_status lossGrad(hase_proposal* net, DeviceBatch& d, uint32_t g0, uint32_t g1, float* dLoss, float* dGrad) {
    const uint32_t r0 = d.offsets[g0], r1 = d.offsets[g1];
    const uint32_t rows = r1 - r0;
    if (rows == 0) return HASE_OK;
    const uint32_t tiles = (rows + kTile - 1) / kTile;
    const uint32_t grid = std::min(tiles, 2u * net->numSMs);  // two CTAs per SM
    const uint32_t fgrid = std::min(tiles, net->numSMs * kMlpBlocksPerSM);
    ForwardLaunch F{net->wimg.p, net->vec.p, d.features.p + size_t(r0) * kFeat, d.logits.p + r0, rows, net->error.p};
    mlpForwardKernel<<<fgrid, kTile, kSmemBytes, net->stream>>>(F);
    HASE_CUDA(cudaGetLastError());
    StatsLaunch S{d.logits.p, d.targets.p, d.hasWeights ? d.weights.p : nullptr, d.doffsets.p, g0, 0u,
                  1.0f / float(g1 - g0), d.dl.p, dLoss};
    groupStatsKernel<<<g1 - g0, 256, 0, net->stream>>>(S);
    HASE_CUDA(cudaGetLastError());
    TrainLaunch T{net->wimg.p, net->vec.p, d.features.p + size_t(r0) * kFeat, d.dl.p + r0, rows, dGrad,
                  net->error.p};
    mlpBackwardKernel<<<grid, kTile, kTrainSmemBytes, net->stream>>>(T);
    HASE_CUDA(cudaGetLastError());
    return HASE_OK;
}

hase_status prepareTraining(hase_proposal* net) {
    HASE_CUDA(cudaSetDevice(net->device));
    HASE_CUDA(cudaFuncSetAttribute(mlpForwardKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemBytes)));
    HASE_CUDA(
        cudaFuncSetAttribute(mlpBackwardKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kTrainSmemBytes)));
    HASE_CUDA(net->grad.ensure(HASE_PROPOSAL_PARAMS));
    HASE_CUDA(net->loss.ensure(1));
    return HASE_OK;
}

}  // namespace

extern "C" {

hase_status hase_proposal_loss_grad(hase_proposal* net, const hase_proposal_batch* batch, float* loss, float* grad) {
    if (!net || !loss || !grad) return fail(HASE_INVALID_ARGUMENT, "null argument");
    HASE_TRY(prepareTraining(net));
    DeviceBatch d;
    HASE_TRY(uploadBatch(net, batch, d));
    HASE_CUDA(cudaMemsetAsync(net->grad.p, 0, HASE_PROPOSAL_PARAMS * sizeof(float), net->stream));
    HASE_CUDA(cudaMemsetAsync(net->loss.p, 0, sizeof(float), net->stream));
    HASE_TRY(lossGrad(net, d, 0, d.groups, net->loss.p, net->grad.p));
    HASE_CUDA(cudaMemcpyAsync(grad, net->grad.p, HASE_PROPOSAL_PARAMS * sizeof(float), cudaMemcpyDeviceToHost,
                              net->stream));
    HASE_CUDA(cudaMemcpyAsync(loss, net->loss.p, sizeof(float), cudaMemcpyDeviceToHost, net->stream));
    HASE_CUDA(cudaStreamSynchronize(net->stream));
    return checkError(net);
}

hase_status hase_proposal_train(hase_proposal* net, const hase_proposal_batch* batch,
                                const hase_proposal_train_desc* tr, float* lossHistory) {
    if (!net || !tr) return fail(HASE_INVALID_ARGUMENT, "null argument");
    if (tr->steps == 0) return HASE_OK;
    if (tr->groupsPerStep == 0) return fail(HASE_INVALID_ARGUMENT, "groupsPerStep must be positive");
    if (!(tr->learningRate > 0.0f)) return fail(HASE_INVALID_ARGUMENT, "learningRate must be positive");
    HASE_TRY(prepareTraining(net));
    DeviceBatch d;
    HASE_TRY(uploadBatch(net, batch, d));
    if (tr->groupsPerStep > d.groups) return fail(HASE_INVALID_ARGUMENT, "groupsPerStep exceeds the groups");
    const float b1 = tr->beta1 > 0.0f ? tr->beta1 : 0.9f, b2 = tr->beta2 > 0.0f ? tr->beta2 : 0.999f;
    const float eps = tr->epsilon > 0.0f ? tr->epsilon : 1e-8f;
    DevBuf<float> hist;
    HASE_CUDA(hist.ensure(tr->steps));
    HASE_CUDA(cudaMemsetAsync(hist.p, 0, tr->steps * sizeof(float), net->stream));
    HASE_CUDA(net->dparams.ensure(HASE_PROPOSAL_PARAMS));
    HASE_CUDA(net->adamM.ensure(HASE_PROPOSAL_PARAMS));
    HASE_CUDA(net->adamV.ensure(HASE_PROPOSAL_PARAMS));
    HASE_CUDA(cudaMemcpyAsync(net->dparams.p, net->params.data(), HASE_PROPOSAL_PARAMS * sizeof(float),
                              cudaMemcpyHostToDevice, net->stream));
    HASE_CUDA(cudaMemsetAsync(net->adamM.p, 0, HASE_PROPOSAL_PARAMS * sizeof(float), net->stream));
    HASE_CUDA(cudaMemsetAsync(net->adamV.p, 0, HASE_PROPOSAL_PARAMS * sizeof(float), net->stream));
    const uint32_t blocks = d.groups / tr->groupsPerStep;
    double p1 = 1.0, p2 = 1.0;
    for (uint32_t step = 0; step < tr->steps; ++step) {
        const uint32_t g0 = (step % blocks) * tr->groupsPerStep, g1 = g0 + tr->groupsPerStep;
        HASE_CUDA(cudaMemsetAsync(net->grad.p, 0, HASE_PROPOSAL_PARAMS * sizeof(float), net->stream));
        HASE_TRY(lossGrad(net, d, g0, g1, hist.p + step, net->grad.p));
        p1 *= b1;
        p2 *= b2;
        adamKernel<<<(HASE_PROPOSAL_PARAMS + 255) / 256, 256, 0, net->stream>>>(
            net->dparams.p, net->adamM.p, net->adamV.p, net->grad.p, HASE_PROPOSAL_PARAMS, tr->learningRate, b1, b2,
            eps, float(1.0 - p1), float(1.0 - p2));
        packKernel<<<(kPackThreads + 255) / 256, 256, 0, net->stream>>>(
            net->dparams.p, reinterpret_cast<uint8_t*>(net->wimg.p), net->vec.p);
        HASE_CUDA(cudaGetLastError());
    }
    HASE_CUDA(cudaMemcpyAsync(net->params.data(), net->dparams.p, HASE_PROPOSAL_PARAMS * sizeof(float),
                              cudaMemcpyDeviceToHost, net->stream));
    if (lossHistory)
        HASE_CUDA(cudaMemcpyAsync(lossHistory, hist.p, tr->steps * sizeof(float), cudaMemcpyDeviceToHost, net->stream));
    HASE_CUDA(cudaStreamSynchronize(net->stream));
    return checkError(net);
}

}  // extern "C"
