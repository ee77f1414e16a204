// hase_b200.cu -- libhase_b200.so: sm_100a kernels of the backward,
// importance-sampled phi-ASE method and the C ABI around them.
//
// Per batch of sample points (prism mesh, FP32 geometry, FP64 sums):
//   (a1) importanceKernel  one thread per (sample, reflection slice, prism):
//        straight-line walk from the prism centre to the (image) sample point,
//        ln w = ln(beta V / d^2) + Int g dl.
//   (a2) mapKernel         one CTA per sample: w = exp(ln w - max), integer
//        quantisation q = ceil(w 2^24 / max w), warp-shuffle scans of q over
//        one contiguous segment per warp and the systematic-sampling ray offsets
//        offsets[b] = floor((C_b M + floor(phase Q / 2^32)) / Q).
//   (b)  rayKernel         CTAs over (ray chunk, active sample): Philox4x32-10
//        start points, prism walk (neighbour + level crossings, top/bottom
//        reflections), per-ray X = N_tot/(4 pi tau) beta V (Q/q) exp(G)/d^2,
//        warp-shuffle FP64 reduction of sum X and sum X^2 per chunk.
//   (c/d) finalizeKernel   one warp per active sample: deterministic reduction
//        of the chunk partials, phi = sum/N, relative error, and compaction of
//        the samples still above the threshold for the next adaptive pass.
// Reference anchors (HASEonGPU v2.2.0 tree): result/experiment types
// include/core/types.hpp:201-354; dndt include/core/forwardPhiAseUtilities.hpp:16-25;
// entry point include/core/simulation.hpp:42-47.
#include "hase_b200.h"
#include "hase_b200_batch.h"
#include "hase_b200_forward.h"
#include "hase_b200_proposal.h"
#include "hase_device.cuh"
#include "hase_host.cuh"
#include "hase_mlp.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <limits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

using namespace hase;

namespace hase {

thread_local std::string g_lastError;

hase_status fail(hase_status st, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_lastError = buf;
    return st;
}

}  // namespace hase

namespace {

constexpr uint32_t kRayBlock = 256;
constexpr int kRayMinBlocks = 5;
constexpr int kRefill = 8;  // idle lanes that trigger a batched refill
constexpr uint32_t kMaxItems = 1024;  // work items per sample and pass
constexpr uint32_t kMinItemRays = 1024;
constexpr uint32_t kMapBlock = 1024;
#ifndef HASE_WALK_COLUMNS
#define HASE_WALK_COLUMNS 32
#endif
constexpr int kWalkColumns = HASE_WALK_COLUMNS;  // triangle columns per stepRay call of the ray kernel
constexpr double kPi = 3.14159265358979323846;

// ------------------------------------------------------------ reductions ----
template <typename T>
__device__ __forceinline__ T warpSum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float warpMax(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Warp-wide inclusive scan.
template <typename T>
__device__ __forceinline__ T warpInclusiveScan(T v) {
    const uint32_t lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= uint32_t(o)) v += n;
    }
    return v;
}

// --------------------------------------------------------- (a1) weights ----
struct ImportanceLaunch {
    MeshView m;
    uint32_t firstSample, slices, nW;
    float A, B;   // spectrally averaged gain coefficients
    float* lnw;   // [rows][nW]
    const uint32_t* rowList;  // rows to compute (blockIdx.y indexes it), or null: rows 0 .. gridDim.y - 1
    const uint8_t* rowFlag;   // batched media: only rows with rowFlag[flagBase + row] set are computed (or null)
    uint32_t flagBase;
    unsigned long long* crossings;  // counting launches only: total walk crossings
    // local proposal: the K candidate triangles of every point ([Np][K]); the
    // row then holds slices x layers x K entries (j (layers K) + l K + k)
    const uint32_t* cand;
    uint32_t K;
};

// One thread per (sample, reflection slice, triangle, group of G layers): the
// straight lines from the centres of the G prisms (t, l) to the (image)
// sample point all project onto the same 2-D segment, centroid -> sample
// point, so they cross the same triangles at the same 2-D distances sigma.
// The thread walks that 2-D segment once (edge tests shared by the G lines)
// and, per line, the level planes and top/bottom reflections inside each
// triangle: plane k of line l lies at sigma = D2 (k - kImg) / (l + 1/2 - kImg).
// ln w = ln(beta V / d^2) + Int g dl, Int g dl = (D3 / D2) Int g dsigma.
// TAB: g of every prism is read from m.gTab (built for L.A, L.B) instead of
// being evaluated from beta at every crossing.
template <int G, bool TAB = false>
__global__ void __launch_bounds__(256) importanceKernel(ImportanceLaunch L) {
    const MeshView& m = L.m;
    const float* gcol = TAB ? m.gTab : m.gainBeta;
    const uint32_t groups = (m.layers + G - 1) / G;
    const uint32_t perSlice = groups * m.T;
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= L.slices * perSlice) return;
    const uint32_t row = L.rowList ? L.rowList[blockIdx.y] : blockIdx.y;
    if (L.rowFlag && !L.rowFlag[L.flagBase + row]) return;
    const uint32_t j = idx / perSlice;
    const uint32_t rem = idx - j * perSlice;
    const uint32_t grp = rem / m.T, t = rem - grp * m.T;
    const int l0 = int(grp * G);
    const uint32_t sample = L.firstSample + row;
    const float2 S = __ldg(m.points + sample % m.Np);
    const int ls = int(sample / m.Np);
    const int kImg = imageLevel(ls, int(m.layers), j);
    const float2 c = __ldg(m.centroid + t);
    const float area = __ldg(&m.geo[2 * t + 1].z);
    const float dx = c.x - S.x, dy = c.y - S.y;
    const float D2 = sqrtf(fmaf(dx, dx, dy * dy));
    const float inv2 = 1.0f / D2;
    const float ux = dx * inv2, uy = dy * inv2;
    float* out = L.lnw + size_t(row) * L.nW + size_t(j) * m.P + t;

    float J[G], lnR[G], invc[G];
    // the line's next level plane lies at s = kf * invc: kf is the plane's
    // level offset from the image level (an exact small-integer float) and
    // invc the distance per level, both times the line's layer step toward the
    // image level, so that kf grows by 1 per plane
    float kf[G];
    // lrow: the line's physical layer x T; rstep: the row offset of the next
    // physical layer toward the image level (+-T, flipped at a reflection)
    int lrow[G], rstep[G], left[G];
    bool ok[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
        const int l = l0 + g;
        ok[g] = l < int(m.layers) && __ldg(m.srcBeta + size_t(min(l, int(m.layers) - 1)) * m.T + t) > 0.0f;
        J[g] = 0.0f;
        lnR[g] = 0.0f;
        kf[g] = kImg > l ? float(l + 1 - kImg) : float(kImg - l);
        lrow[g] = l * int(m.T);
        rstep[g] = kImg > l ? int(m.T) : -int(m.T);
        left[g] = expectedReflections(j);
        const float ic = D2 / (float(l - kImg) + 0.5f);
        invc[g] = kImg > l ? ic : -ic;
    }
    GlobalLoader load{m.walk};
    uint32_t tk = t;
    float sc = D2;
    bool done = false;
    for (int step = 0; step < kMaxSteps && !done; ++step) {
        float4 a, b, cc;
        load(tk, a, b, cc);
        float bn = -1.0f, bd = 0.0f;
        int bw = -1;
        const auto edge = [&](float nx, float ny, float ce, int nbw) {
            const float dd = -fmaf(nx, ux, ny * uy);
            const float nm = fmaf(nx, S.x, fmaf(ny, S.y, -ce));
            const bool okE = dd > 0.0f;  // the entry edge has dd < 0, a boundary edge NaN (see stepRay)
            if (okE && nm * bd > bn * dd) {
                bn = nm;
                bd = dd;
                bw = nbw;
            }
        };
        edge(a.x, a.y, a.z, __float_as_int(cc.y));
        edge(a.w, b.x, b.y, __float_as_int(cc.z));
        edge(b.z, b.w, cc.x, __float_as_int(cc.w));
        float sOut = fmaxf(fminf(__fdividef(bn, bd), sc), 0.0f);
        if (sOut <= m.tolEnd) {
            sOut = 0.0f;
            done = true;
        }
        // beta of every line's current prism in this triangle, issued together
        float gbv[G];
#pragma unroll
        for (int g = 0; g < G; ++g) gbv[g] = ok[g] ? __ldg(gcol + uint32_t(lrow[g]) + tk) : 0.0f;
#pragma unroll
        for (int g = 0; g < G; ++g) {
            if (!ok[g]) continue;
            float s = sc;
            float gb = gbv[g];
            while (true) {
                const float sb = kf[g] * invc[g];
                if (!(sb > sOut)) break;
                J[g] = fmaf(TAB ? gb : ((gb == gb) ? fmaf(gb, L.A, -L.B) : -m.cladAbs), s - sb, J[g]);
                s = sb;
                const int cand = lrow[g] + rstep[g];
                if (uint32_t(cand) >= m.P) {  // a physical bottom/top surface: reflect
                    if (left[g] <= 0) {
                        ok[g] = false;
                        break;
                    }
                    const float dz = (float(l0 + g - kImg) + 0.5f) * m.h;
                    const float uz = dz * rsqrtf(fmaf(D2, D2, dz * dz));
                    lnR[g] += __logf(reflectFactor(m, tk, cand < 0 ? 0 : 1, uz));
                    --left[g];
                    rstep[g] = -rstep[g];
                } else {
                    lrow[g] = cand;
                    gb = __ldg(gcol + uint32_t(cand) + tk);
                }
                kf[g] += 1.0f;
            }
            if (!ok[g]) continue;
            J[g] = fmaf(TAB ? gb : ((gb == gb) ? fmaf(gb, L.A, -L.B) : -m.cladAbs), s - sOut, J[g]);
        }
        if (!done) {
            tk = uint32_t(bw) >> 2;
            sc = sOut;
        }
    }
#pragma unroll
    for (int g = 0; g < G; ++g) {
        const int l = l0 + g;
        if (l >= int(m.layers)) continue;
        float v = -INFINITY;
        if (ok[g] && done) {
            const float dz = (float(l - kImg) + 0.5f) * m.h;
            const float D3sq = fmaf(D2, D2, dz * dz);
            if (left[g] > 0) {  // the bounce happens at the target itself, in the final triangle
                lnR[g] += __logf(reflectFactor(m, tk, lrow[g] + rstep[g] < 0 ? 0 : 1, dz * rsqrtf(D3sq)));
            }
            const float beta = __ldg(m.srcBeta + size_t(l) * m.T + t);
            v = __logf(beta * area * m.h / D3sq) + J[g] * (sqrtf(D3sq) * inv2) + lnR[g];
        }
        out[size_t(l) * m.T] = v;
    }
}

// Line-team importance kernel: a team of TL lanes per (sample row,
// triangle t).  Every line from the centre of a prism (t, l) to an image
// s_j of the sample point projects onto the same 2-D segment, centroid ->
// sample point, so the team walks that segment in lock step (no divergence
// in the number of triangles crossed) and each lane carries LPL of the
// triangle's slices x layers lines through the level planes and
// reflections of every triangle on it (teams of TL lanes, lines in chunks
// of TL x LPL).  The 2-D edge tests are thus shared by up to TL x LPL lines
// instead of the G of importanceKernel; the per-line arithmetic is
// importanceKernel's, operation for operation, so the weights are the same
// bits.  COUNT: also add the walk's crossings (triangle segments plus level
// planes and reflections, per line) to *L.crossings.
template <int TL, int LPL, bool TAB = false, bool COUNT = false>
__global__ void __launch_bounds__(256) importanceTeamKernel(ImportanceLaunch L) {
    static_assert(TL >= 1 && TL <= 32 && (32 % TL) == 0, "a team is a power-of-two part of a warp");
    const MeshView& m = L.m;
    const float* gcol = TAB ? m.gTab : m.gainBeta;
    constexpr uint32_t kTeams = 256 / TL;
    const uint32_t tIdx = blockIdx.x * kTeams + threadIdx.x / TL;  // triangle (or candidate) of the team
    const uint32_t li = threadIdx.x % TL;
    const uint32_t row = L.rowList ? L.rowList[blockIdx.y] : blockIdx.y;
    const uint32_t strideL = L.cand ? L.K : m.T;            // entries per layer of a slice
    unsigned long long counted = 0;
    if (tIdx < strideL && !(L.rowFlag && !L.rowFlag[L.flagBase + row])) {
        const uint32_t sample = L.firstSample + row;
        const uint32_t pt = sample % m.Np;
        const uint32_t t = L.cand ? __ldg(L.cand + size_t(pt) * L.K + tIdx) : tIdx;
        const float2 S = __ldg(m.points + pt);
        const int ls = int(sample / m.Np);
        const float2 c = __ldg(m.centroid + t);
        const float area = __ldg(&m.geo[2 * t + 1].z);
        const float dx = c.x - S.x, dy = c.y - S.y;
        const float D2 = sqrtf(fmaf(dx, dx, dy * dy));
        const float inv2 = 1.0f / D2;
        const float ux = dx * inv2, uy = dy * inv2;
        float* outRow = L.lnw + size_t(row) * L.nW + tIdx;
        const size_t strideJ = size_t(strideL) * m.layers;
        const uint32_t nLines = L.slices * m.layers;
        for (uint32_t c0 = 0; c0 < nLines; c0 += TL * LPL) {
            float J[LPL], lnR[LPL], invc[LPL], nextPlane[LPL];
            float kf[LPL];  // as in importanceKernel
            int lrow[LPL], rstep[LPL], left[LPL], kImg[LPL], lay[LPL];  // lrow, rstep: as in importanceKernel
            uint32_t sl[LPL];
            bool ok[LPL];
            const uint16_t* order = m.lineOrder[L.slices == 5 ? 1 : 0];
#pragma unroll
            for (int g = 0; g < LPL; ++g) {
                const uint32_t qq = c0 + li + uint32_t(TL * g);
                const bool valid = qq < nLines;
                const uint32_t q = valid && order ? uint32_t(__ldg(order + size_t(ls) * nLines + qq)) : qq;
                const uint32_t l = valid ? q / L.slices : 0u;
                const uint32_t j = valid ? q - l * L.slices : 0u;
                sl[g] = valid ? j : 0xffffffffu;
                lay[g] = int(l);
                kImg[g] = imageLevel(ls, int(m.layers), j);
                ok[g] = valid && __ldg(m.srcBeta + size_t(l) * m.T + t) > 0.0f;
                J[g] = 0.0f;
                lnR[g] = 0.0f;
                kf[g] = kImg[g] > int(l) ? float(int(l) + 1 - kImg[g]) : float(kImg[g] - int(l));
                lrow[g] = int(l * m.T);
                rstep[g] = kImg[g] > int(l) ? int(m.T) : -int(m.T);
                left[g] = expectedReflections(j);
                const float ic = D2 / (float(int(l) - kImg[g]) + 0.5f);
                invc[g] = kImg[g] > int(l) ? ic : -ic;
                // sigma of the next level plane toward the image level (carried,
                // recomputed only when the line crosses it)
                nextPlane[g] = kf[g] * invc[g];
            }
            GlobalLoader load{m.walk};
            uint32_t tk = t;
            float sc = D2;
            bool done = false;
            for (int step = 0; step < kMaxSteps && !done; ++step) {
                float4 a, b, cc;
                load(tk, a, b, cc);
                float bn = -1.0f, bd = 0.0f;
                int bw = -1;
                const auto edge = [&](float nx, float ny, float ce, int nbw) {
                    const float dd = -fmaf(nx, ux, ny * uy);
                    const float nm = fmaf(nx, S.x, fmaf(ny, S.y, -ce));
                    const bool okE = dd > 0.0f;  // the entry edge has dd < 0, a boundary edge NaN (see stepRay)
                    if (okE && nm * bd > bn * dd) {
                        bn = nm;
                        bd = dd;
                        bw = nbw;
                    }
                };
                edge(a.x, a.y, a.z, __float_as_int(cc.y));
                edge(a.w, b.x, b.y, __float_as_int(cc.z));
                edge(b.z, b.w, cc.x, __float_as_int(cc.w));
                float sOut = fmaxf(fminf(__fdividef(bn, bd), sc), 0.0f);
                if (sOut <= m.tolEnd) {
                    sOut = 0.0f;
                    done = true;
                }
                float gbv[LPL];
#pragma unroll
                for (int g = 0; g < LPL; ++g) gbv[g] = ok[g] ? __ldg(gcol + uint32_t(lrow[g]) + tk) : 0.0f;
#pragma unroll
                for (int g = 0; g < LPL; ++g) {
                    if (!ok[g]) continue;
                    if (COUNT) ++counted;
                    float s = sc;
                    float gb = gbv[g];
                    while (true) {
                        const float sb = nextPlane[g];
                        if (!(sb > sOut)) break;
                        if (COUNT) ++counted;
                        J[g] = fmaf(TAB ? gb : ((gb == gb) ? fmaf(gb, L.A, -L.B) : -m.cladAbs), s - sb, J[g]);
                        s = sb;
                        const int cand = lrow[g] + rstep[g];
                        if (uint32_t(cand) >= m.P) {  // a physical bottom/top surface: reflect
                            if (left[g] <= 0) {
                                ok[g] = false;
                                break;
                            }
                            const float dz = (float(lay[g] - kImg[g]) + 0.5f) * m.h;
                            const float uz = dz * rsqrtf(fmaf(D2, D2, dz * dz));
                            lnR[g] += __logf(reflectFactor(m, tk, cand < 0 ? 0 : 1, uz));
                            --left[g];
                            rstep[g] = -rstep[g];
                        } else {
                            lrow[g] = cand;
                            gb = __ldg(gcol + uint32_t(cand) + tk);
                        }
                        kf[g] += 1.0f;
                        nextPlane[g] = kf[g] * invc[g];
                    }
                    if (!ok[g]) continue;
                    J[g] = fmaf(TAB ? gb : ((gb == gb) ? fmaf(gb, L.A, -L.B) : -m.cladAbs), s - sOut, J[g]);
                }
                if (!done) {
                    tk = uint32_t(bw) >> 2;
                    sc = sOut;
                }
            }
#pragma unroll
            for (int g = 0; g < LPL; ++g) {
                if (sl[g] == 0xffffffffu) continue;
                const int l = lay[g];
                float v = -INFINITY;
                if (ok[g] && done) {
                    const float dz = (float(l - kImg[g]) + 0.5f) * m.h;
                    const float D3sq = fmaf(D2, D2, dz * dz);
                    if (left[g] > 0) {  // the bounce happens at the target itself, in the final triangle
                        lnR[g] += __logf(reflectFactor(m, tk, lrow[g] + rstep[g] < 0 ? 0 : 1, dz * rsqrtf(D3sq)));
                    }
                    const float beta = __ldg(m.srcBeta + size_t(l) * m.T + t);
                    v = __logf(beta * area * m.h / D3sq) + J[g] * (sqrtf(D3sq) * inv2) + lnR[g];
                }
                outRow[size_t(sl[g]) * strideJ + size_t(l) * strideL] = v;
            }
        }
    }
    if (COUNT) {
        counted = warpSum(counted);
        if ((threadIdx.x & 31) == 0 && counted) atomicAdd(L.crossings, counted);
    }
}

// Team width of the line-team kernel: the narrowest team whose lanes hold a
// sample's slices x layers lines of one triangle in one chunk of 3 per lane
// (32 lanes: chunks of 96 lines).
uint32_t importanceTeamWidth(uint32_t lines) {
    return lines <= 12 ? 4u : lines <= 24 ? 8u : lines <= 48 ? 16u : 32u;
}

// The importance walks of `rows` sample rows: layers = 0 (the library's
// choice): importanceTeamKernel; 2, 4 or 8: importanceKernel with that many
// prism layers per thread.  tab: il.m.gTab holds g for il.A, il.B.  count:
// the counting team kernel (il.crossings accumulates the walk's crossings).
cudaError_t launchImportance(uint32_t layers, const ImportanceLaunch& il, uint32_t meshLayers, uint32_t T,
                             uint32_t rows, cudaStream_t stream, bool tab = false, bool count = false) {
    if (layers == 0 || count || il.cand) {
        const uint32_t tl = importanceTeamWidth(il.slices * meshLayers);
        const uint32_t nTri = il.cand ? il.K : T;
#define HASE_TEAM(TL)                                                                         \
    {                                                                                         \
        const dim3 grid((nTri + 256 / TL - 1) / (256 / TL), rows);                            \
        if (count) importanceTeamKernel<TL, 3, false, true><<<grid, 256, 0, stream>>>(il);   \
        else if (tab) importanceTeamKernel<TL, 3, true><<<grid, 256, 0, stream>>>(il);       \
        else importanceTeamKernel<TL, 3><<<grid, 256, 0, stream>>>(il);                      \
    }
        switch (tl) {
            case 4: HASE_TEAM(4) break;
            case 8: HASE_TEAM(8) break;
            case 16: HASE_TEAM(16) break;
            default: HASE_TEAM(32) break;
        }
#undef HASE_TEAM
        return cudaGetLastError();
    }
    const uint32_t G = layers;
    const uint32_t threads = il.slices * ((meshLayers + G - 1) / G) * T;
    const dim3 grid((threads + 255) / 256, rows);
    if (G == 2) {
        if (tab) importanceKernel<2, true><<<grid, 256, 0, stream>>>(il);
        else importanceKernel<2><<<grid, 256, 0, stream>>>(il);
    } else if (G == 8) {
        if (tab) importanceKernel<8, true><<<grid, 256, 0, stream>>>(il);
        else importanceKernel<8><<<grid, 256, 0, stream>>>(il);
    } else {
        if (tab) importanceKernel<4, true><<<grid, 256, 0, stream>>>(il);
        else importanceKernel<4><<<grid, 256, 0, stream>>>(il);
    }
    return cudaGetLastError();
}

bool validImportanceLayers(uint32_t layers) {
    return layers == 0 || layers == 2 || layers == 4 || layers == 8;
}

// ------------------------------------------------- batched gain media ----
// One medium of a batched solve (device array, one entry per instance).
struct InstanceView {
    MeshView m;
    const float2* spec;           // per wavelength (A, B)
    uint32_t nLambda, nW, seedLo, pad;
    double C;                     // N_tot / (4 pi tau)
};

// One sample row of a batched solve: its [rows][nW] workspace arrays start at
// element w (the [rows][nW + 1] offsets at w + row index).
struct RowInfo {
    unsigned long long w;
    uint32_t inst, sample, nW, seedLo;
};

// ------------------------------------------------------- (a2) ray map ----
struct MapLaunch {
    const float* in;            // [rows][nW]: ln w (isLog) or w
    int isLog;
    int full;                   // 1: quantise + Q; 0: reuse q, Q
    const uint32_t* rowList;    // nullptr: row = block index
    uint32_t nW;
    uint32_t M;                 // rays to map this pass
    const uint32_t* phases;     // nullptr: Philox(0, sample, pass, map tag)
    uint32_t firstSample, pass, seedLo, seedHi;
    float* wOut;                // optional [rows][nW] normalised weights
    uint32_t* q;                // [rows][nW]
    unsigned long long* Q;      // [rows]
    uint32_t* offsets;          // [rows][nW+1]
    const RowInfo* rows;        // batched media: ragged rows (nW, workspace offset, sample, seed per row)
    const unsigned int* count;  // batched media: rows of rowList to map (device), blocks stride over them
    const uint8_t* rowFlag;     // batched media: only rows with rowFlag[row] set are mapped (or null)
};

// Each warp owns one contiguous segment of the row (a multiple of 32 entries
// long, the last one cut at nW): the passes read and write it coalesced, four
// loads in flight per lane, and the offsets' prefix sums need one block-wide
// step (the warps' exclusive prefixes) instead of a block scan per 1,024
// entries.  q, Q and the offsets are integers, so they do not depend on the
// order of the sums.
__device__ void mapRow(const MapLaunch& L, uint32_t row) {
    constexpr uint32_t kWarps = kMapBlock / 32;
    static_assert(kWarps == 32, "one warp prefix per lane");
    __shared__ unsigned long long sWarp[kWarps];  // q sum of each warp's segment, then its exclusive prefix
    __shared__ float sMax;
    __shared__ unsigned long long sQ;
    __shared__ float sRed[kWarps];
    uint32_t nW = L.nW, sample = L.firstSample + row, seedLo = L.seedLo;
    size_t wBase = size_t(row) * nW, oBase = size_t(row) * (nW + 1);
    if (L.rows) {
        const RowInfo ri = L.rows[row];
        nW = ri.nW;
        sample = ri.sample;
        seedLo = ri.seedLo;
        wBase = ri.w;
        oBase = ri.w + row;
    }
    const float* in = L.in + wBase;
    uint32_t* q = L.q + wBase;
    uint32_t* off = L.offsets + oBase;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t segLen = ((nW + kWarps - 1) / kWarps + 31u) & ~31u;
    const uint32_t s0 = min(nW, warp * segLen), s1 = min(nW, s0 + segLen);
    unsigned long long part = 0;
    if (L.full) {
        float mx = -INFINITY;
        {
            uint32_t b = s0 + lane;
            for (; b + 96 < s1; b += 128)
                mx = fmaxf(fmaxf(mx, fmaxf(in[b], in[b + 32])), fmaxf(in[b + 64], in[b + 96]));
            for (; b < s1; b += 32) mx = fmaxf(mx, in[b]);
        }
        mx = warpMax(mx);
        if (lane == 0) sRed[warp] = mx;
        __syncthreads();
        if (warp == 0) {
            const float v = warpMax(sRed[lane]);
            if (lane == 0) sMax = v;
        }
        __syncthreads();
        mx = sMax;
        // Normalised weights: exp(ln w - max) has maximum exactly 1.
        const float wmax = L.isLog ? (mx == -INFINITY ? 0.0f : 1.0f) : mx;
        const double scale = wmax > 0.0f ? 16777216.0 / double(wmax) : 0.0;
        const auto quantise = [&](uint32_t b, float v) {
            const float w = L.isLog ? (v == -INFINITY || wmax == 0.0f ? 0.0f : expf(v - mx)) : v;
            const uint32_t qi = (w > 0.0f && wmax > 0.0f) ? uint32_t(ceil(double(w) * scale)) : 0u;
            q[b] = qi;
            if (L.wOut) L.wOut[wBase + b] = w;
            part += qi;
        };
        uint32_t b = s0 + lane;
        for (; b + 96 < s1; b += 128) {
            const float v0 = in[b], v1 = in[b + 32], v2 = in[b + 64], v3 = in[b + 96];
            quantise(b, v0);
            quantise(b + 32, v1);
            quantise(b + 64, v2);
            quantise(b + 96, v3);
        }
        for (; b < s1; b += 32) quantise(b, in[b]);
    } else {
        uint32_t b = s0 + lane;
        for (; b + 96 < s1; b += 128) part += (unsigned long long)(q[b] + q[b + 32]) + q[b + 64] + q[b + 96];
        for (; b < s1; b += 32) part += q[b];
    }
    part = warpSum(part);
    if (lane == 0) sWarp[warp] = part;
    __syncthreads();
    if (warp == 0) {
        const unsigned long long v = sWarp[lane];
        const unsigned long long incl = warpInclusiveScan(v);
        sWarp[lane] = incl - v;
        if (lane == 31) {
            sQ = incl;
            if (L.full) L.Q[row] = incl;
        }
    }
    __syncthreads();
    const unsigned long long Q = L.full ? sQ : L.Q[row];
    const uint32_t M = L.M;
    if (Q == 0) {
        for (uint32_t b = threadIdx.x; b <= nW; b += kMapBlock) off[b] = 0u;
        return;
    }
    uint32_t phase;
    if (L.phases) {
        phase = L.phases[row];
    } else {
        phase = philox4x32_10(0u, sample, L.pass, kTagMap, seedLo, L.seedHi).x;
    }
    using u128 = unsigned __int128;
    const unsigned long long phiQ = (unsigned long long)((u128(phase) * Q) >> 32);
    // floor(x / Q), x = C M + phiQ, without a 128-bit division: the FP64
    // quotient carries a relative error of a few 2^-53, and the true quotient
    // is at most M < 2^32, so the truncated estimate k is off by at most one.
    // Then x - k Q lies in [-Q, 2Q) with Q < 2^56 (q <= 2^24 + 1, nW < 2^31),
    // so its low 64 bits, from wrapping 64-bit products, decide the correction.
    const double invQ = 1.0 / double(Q);
    unsigned long long carry = sWarp[warp];
    const auto offsetOf = [&](uint32_t b, uint32_t v) {
        const uint32_t incl = warpInclusiveScan(v);  // q <= 2^24 + 1: 32 of them fit 32 bits
        if (b < s1) {
            const unsigned long long C = carry + (incl - v);
            unsigned long long k = (unsigned long long)(fma(double(C), double(M), double(phiQ)) * invQ);
            const long long r = (long long)(C * M + phiQ - k * Q);
            if (r < 0) --k;
            else if (r >= (long long)Q) ++k;
            off[b] = uint32_t(k);
        }
        carry += __shfl_sync(0xffffffffu, incl, 31);
    };
    // warp-uniform trip counts: every lane takes part in the scans
    for (uint32_t base = s0; base < s1; base += 128) {
        const uint32_t b = base + lane;
        const uint32_t v0 = b < s1 ? q[b] : 0u, v1 = b + 32 < s1 ? q[b + 32] : 0u;
        const uint32_t v2 = b + 64 < s1 ? q[b + 64] : 0u, v3 = b + 96 < s1 ? q[b + 96] : 0u;
        offsetOf(b, v0);
        offsetOf(b + 32, v1);
        offsetOf(b + 64, v2);
        offsetOf(b + 96, v3);
    }
    if (threadIdx.x == 0) off[nW] = M;
}

// One CTA per row (grid = rows), or, with L.count, CTAs striding over the
// device-held number of rows.
__global__ void __launch_bounds__(kMapBlock, 2) mapKernel(MapLaunch L) {
    const uint32_t n = L.count ? *L.count : gridDim.x;
    for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const uint32_t row = L.rowList ? L.rowList[i] : i;
        if (L.rowFlag && !L.rowFlag[row]) continue;  // uniform over the block
        mapRow(L, row);
        __syncthreads();  // shared scratch is reused by the next row
    }
}

// --------------------------------------------------------- (b) rays ----
// The far prior of the local proposal: R_j beta V e^Ghat / d^2 over all
// (slice j, prism) pairs, with d a softened distance from the image of the
// sample point in slice j to the prism's cell of a 2-D grid of triangle
// cells at the prism's layer, R_j the slice's reflection factor (1 for the
// direct slice; per bounce, 1 where the line from the cell meets the surface
// beyond its critical angle, else the surface's mean reflectivity), and Ghat = d (g_cl + g_s + 6 g_mid) / 8 an estimate of
// the gain along the way (g_cl: mean g of the cell's prisms of the layer,
// g_s: g of the prism next to the sample point, g_mid: mean over 6 interior
// points of the 2-D segment from the sample point to the cell of the
// layer-averaged coarse gain grid, one value per (row, cell) kept in gMid;
// clamped to [-10, 30]).
// Drawn in three steps: a (cell, slice) pair from the row's prefix of w_cj
// = sum_l term_clj, a layer by a scan of the same terms, a triangle of the
// cell from the cell's beta V prefix of that layer.  p_far(j, t, l) =
// term_clj(beta V) / W, W = sum_cj w_cj, the same expression wherever it is
// evaluated.
struct FarSlices {
    float R[2];    // per surface (bottom, top): mean reflectivity, at least 1/4
    float tir[2];  // per surface: total internal reflection when uz^2 <= tir (0: none)
};

struct FarView {
    const uint32_t* cellOf;     // [T] cell of each triangle
    const uint32_t* cellStart;  // [C + 1] cell segments of cellTris
    const uint32_t* cellTris;   // [T] triangles grouped by cell, ascending within a cell
    const float4* cell;         // [C] (x, y, softening^2, 0)
    const float* cellMass;      // [C][layers] beta V of the cell's prisms of each layer
    const float* triPrefix;     // [layers][T] in cellTris order: inclusive beta V prefix within the cell
    const float* gCell;         // [C][layers] mean g of the cell's prisms of each layer (this solve)
    const double* rowCdf;       // [rows][C][slices] inclusive prefix of the row's (cell, slice) weights
    const float* gMid;          // [rows][C] g_mid of the row's sample point and each cell
    uint32_t C, slices;
    FarSlices refl;
};

__device__ __forceinline__ float farDistance2(float4 cell, float2 S, int l, int kImg, float h) {
    const float dx = cell.x - S.x, dy = cell.y - S.y, dz = (float(l - kImg) + 0.5f) * h;
    return fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, cell.z)));
}

// R_j of a term of slice j whose cell lies dl + 1/2 layers above the image
// level (d2: its squared distance; uz^2 = dz^2 / d2).
__device__ __forceinline__ float farSliceFactor(const FarSlices& S, uint32_t j, int dl, float h, float d2) {
    if (j == 0) return 1.0f;
    const float dz = (float(dl) + 0.5f) * h, dz2 = dz * dz;
    const float rb = dz2 <= S.tir[0] * d2 ? 1.0f : S.R[0];
    const float rt = dz2 <= S.tir[1] * d2 ? 1.0f : S.R[1];
    return j == 1 ? rb : (j == 2 ? rt : rb * rt);
}

// One term of the far prior: R_j m e^Ghat / d^2, Ghat = gmean d.
__device__ __forceinline__ float farTerm(float prior, float mass, float d2, float gmean) {
    const float G = fminf(fmaxf(gmean * sqrtf(d2), -10.0f), 30.0f);
    return __fdividef(prior * mass * __expf(G), d2);
}

// The far prior's mean g along the way, (g_cl + g_s + 6 g_mid) / 8.
__device__ __forceinline__ float farMeanGain(float gcl, float gs, float gmid) {
    return fmaf(0.75f, gmid, 0.125f * (gcl + gs));
}

// g_s of a sample row: g of the point's nearest candidate triangle at the
// layer above the sample level (below it on the top level).
__device__ __forceinline__ float farSampleGain(const float* gTab, const uint32_t* cand, uint32_t K, uint32_t T,
                                               uint32_t layers, uint32_t pt, int ls) {
    const uint32_t l = min(uint32_t(ls), layers - 1u);
    return __ldg(gTab + size_t(l) * T + __ldg(cand + size_t(pt) * K));
}

struct RayLaunch {
    MeshView m;
    const uint32_t* active;       // active row ids
    uint32_t nActive;
    uint32_t firstSample, pass, M, nW;
    uint32_t itemRays;            // rays per work item
    uint32_t itemsPerRow;         // ceil(M / itemRays) <= kMaxItems
    unsigned int* itemCounter;    // zeroed before the launch
    const uint32_t* q;            // [rows][nW]
    const unsigned long long* Q;  // [rows]
    const uint32_t* offsets;      // [rows][nW+1]
    uint32_t seedLo, seedHi;
    const float2* spec;           // per wavelength (A, B)
    uint32_t nLambda;
    uint32_t nearField;           // solid-angle start points in prisms touching the sample
    double C;                     // N_tot / (4 pi tau)
    double* pSum;                 // [rows][kMaxItems]
    double* pSum2;
    uint32_t* pDrop;
    unsigned long long* pCross;
    float* logBuf;                // [rows][nW]: per-(slice, prism) sum of contributions (LOG kernels only)
    // batched media (POOL kernels): per-row medium, workspace offset, sample
    // and seed; the medium's view; the number of active rows (device)
    const InstanceView* inst;
    const RowInfo* rows;
    const unsigned int* count;
    // local proposal (LOCAL kernels): a mixture of two ray sources.  Rays
    // [0, Mnear) follow the map over the K candidate triangles of the
    // sample's point (entries j (layers K) + l K + k); rays [Mnear, M) are
    // far rays, drawn from the prior beta V / d^2 over the whole medium (a
    // slice uniformly).  Every ray is weighted by the mixture's probability
    // of its (slice, prism), (Mnear q_b / Q + Mfar p_far) / M, so neither
    // source has to exclude the other's prisms.
    const uint32_t* cand;         // [Np][K] candidate triangles, nearest first
    const uint32_t* candSorted;   // [Np][K] the same, ascending
    const uint32_t* candRank;     // [Np][K] position in cand of each candSorted entry
    uint32_t K, Mnear;
    uint32_t slices, divKm, divKs;  // entries of a layer: floor(x / K) = (x * divKm) >> divKs
    float nearShare, farShare;      // Mnear / M, (M - Mnear) / M
    FarView far;
};

__device__ __forceinline__ uint32_t upperBound(const uint32_t* a, uint32_t n, uint32_t x) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a[mid] <= x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Start state of ray r of sample `sample`, drawn in reflection slice j and
// prism p with probability qf / Q (qf: the map's integer weight q of the
// entry, or the local proposal's mixture weight): Philox4x32-10 counter (r,
// sample, pass, kTagRay); a uniform point in the prism, or (nearField) the
// solid-angle start in a prism touching the image point.  No wavelength is
// drawn: the walk keeps the path integrals every wavelength's gain is linear
// in, and the ray's contribution is its gain averaged over the spectrum
// (rayMeanGain); ab is the walk's reference pair (the spectrum's first).
// wf: the ray's weight without C Q, beta V / (d^2 qf)
// (uniform start) or beta alpha L / qf (near field).
// Returns |start - image|^2 (0: the start point is the sample point itself).
__device__ __forceinline__ float startRay(const MeshView& m, uint32_t r, uint32_t j, uint32_t p, uint32_t sample,
                                          float2 S, int ls, uint32_t pass, uint32_t seedLo, uint32_t seedHi,
                                          float2 ab, float qf, uint32_t nearField, Ray& ray, float& wf) {
    // layer by an exact multiply-shift: no integer division per ray
    const uint32_t l = prismLayer(m, p), t = p - l * m.T;
    const Philox4 rnd = philox4x32_10(r, sample, pass, kTagRay, seedLo, seedHi);
    uint32_t k1 = rnd.x >> 8, k2 = rnd.y >> 8;
    if (k1 + k2 + 1u > (1u << 24)) {
        k1 = (1u << 24) - 1u - k1;
        k2 = (1u << 24) - 1u - k2;
    }
    const int kImg = imageLevel(ls, int(m.layers), j);
    float dx, dy, dz, alphaL, D2;
    if (nearField && (int(l) == kImg || int(l) + 1 == kImg) &&
        nearFieldStart(m, t, int(l), kImg, sample % m.Np, S, unit24(rnd.x >> 8), unit24(rnd.z >> 8),
                       unit24(rnd.w >> 8), dx, dy, dz, alphaL)) {
        D2 = initRay(ray, t, int(l), dx, dy, dz, kImg, j, ab.x, ab.y, m);
        wf = __fdividef(__ldg(m.srcBeta + p) * alphaL, qf);
    } else {
        const float u1 = unit24(k1), u2 = unit24(k2), u3 = unit24(rnd.z >> 8);
        const float4 g0 = __ldg(m.geo + 2 * t), g1 = __ldg(m.geo + 2 * t + 1);
        const float x = fmaf(u2, g1.x, fmaf(u1, g0.z, g0.x));
        const float y = fmaf(u2, g1.y, fmaf(u1, g0.w, g0.y));
        D2 = initRay(ray, t, int(l), x - S.x, y - S.y, (float(int(l) - kImg) + u3) * m.h, kImg, j, ab.x, ab.y, m);
        wf = __fdividef(__ldg(m.srcBeta + p) * g1.z * m.h, D2 * qf);
    }
    return D2;
}

// The (slice j, prism p) of ray r of a local-proposal row and its mixture
// weight qf, startRay's divisor: the ray contributes C Qn beta V e^G /
// (d^2 qf), so qf = Qn P_mix = Mnear/M q_b + Mfar/M Qn p_far.  Near rays take
// the map's entry b; far rays draw from the prior (one Philox block: the
// (cell, slice) pair from 53 bits, the layer, the triangle) and look the
// drawn triangle up among the point's candidates for its q_b.  bsel: the prism's
// candidate entry (for the contribution log) or ~0u.  Returns false for a
// ray without a source (qf = 0).
__device__ __forceinline__ bool localSource(const RayLaunch& L, const MeshView& m, uint32_t row, uint32_t sample,
                                            float2 S, uint32_t r, const uint32_t* q, const uint32_t* off,
                                            uint32_t pb, uint32_t count, unsigned long long Qrow,
                                            unsigned long long Qn, uint32_t seedLo, uint32_t& j, uint32_t& p,
                                            float& qf, uint32_t& bsel) {
    const uint32_t pt = sample % m.Np;
    const int ls = int(sample / m.Np);
    const uint32_t layerK = m.layers * L.K;
    const FarView& F = L.far;
    uint32_t t, l, b = 0xffffffffu, cellIdx = 0;
    const float gs = L.farShare > 0.0f ? farSampleGain(m.gTab, L.cand, L.K, m.T, m.layers, pt, ls) : 0.0f;
    j = 0;
    if (r < L.Mnear) {
        if (Qrow == 0ull) return false;  // the map places no near ray in a row without candidate weight
        b = pb + upperBound(off + pb, count, r) - 1u;
        uint32_t rem = b;  // entry j (layers K) + l K + k
        while (rem >= layerK) {
            rem -= layerK;
            ++j;
        }
        l = uint32_t((uint64_t(rem) * L.divKm) >> L.divKs);
        t = __ldg(L.cand + size_t(pt) * L.K + (rem - l * L.K));
        if (L.farShare > 0.0f) cellIdx = __ldg(F.cellOf + t);
    } else {
        const uint32_t nE = F.C * F.slices;
        const double* cdf = F.rowCdf + size_t(row) * nE;
        const double total = __ldg(cdf + nE - 1);
        if (!(total > 0.0)) return false;
        const Philox4 a = philox4x32_10(r, sample, L.pass, kTagFar, seedLo, L.seedHi);
        const double target = double((uint64_t(a.x) << 21) | (a.y >> 11)) * (1.0 / 9007199254740992.0) * total;
        uint32_t lo = 0, hi = nE - 1;  // first (cell, slice) whose inclusive prefix exceeds the target
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(cdf + mid) <= target) lo = mid + 1;
            else hi = mid;
        }
        cellIdx = lo / F.slices;
        j = lo - cellIdx * F.slices;
        const int kImg = imageLevel(ls, int(m.layers), j);
        const float4 cl = __ldg(F.cell + cellIdx);
        const float wc = float(__ldg(cdf + lo) - (lo ? __ldg(cdf + lo - 1) : 0.0));
        const float target2 = unit24(a.z >> 8) * wc;
        const float* mass = F.cellMass + size_t(cellIdx) * m.layers;
        const float* gc = F.gCell + size_t(cellIdx) * m.layers;
        const float gmid = __ldg(F.gMid + size_t(row) * F.C + cellIdx);
        float acc = 0.0f;  // the layer terms of farRowKernel, in its order
        l = 0xffffffffu;
        for (uint32_t l2 = 0; l2 < m.layers; ++l2) {
            const float mcl = __ldg(mass + l2);
            if (!(mcl > 0.0f)) continue;
            const float d2 = farDistance2(cl, S, int(l2), kImg, m.h);
            acc += farTerm(farSliceFactor(F.refl, j, int(l2) - kImg, m.h, d2), mcl, d2,
                           farMeanGain(__ldg(gc + l2), gs, gmid));
            l = l2;
            if (acc > target2) break;
        }
        if (l == 0xffffffffu) return false;
        const uint32_t s0 = __ldg(F.cellStart + cellIdx), s1 = __ldg(F.cellStart + cellIdx + 1);
        const float* pre = F.triPrefix + size_t(l) * m.T;
        const float target3 = unit24(a.w >> 8) * __ldg(pre + s1 - 1);
        uint32_t lo3 = s0, hi3 = s1 - 1;  // first triangle of the cell whose prefix exceeds the target
        while (lo3 < hi3) {
            const uint32_t mid = (lo3 + hi3) >> 1;
            if (__ldg(pre + mid) <= target3) lo3 = mid + 1;
            else hi3 = mid;
        }
        t = __ldg(F.cellTris + lo3);
        if (Qrow != 0ull) {  // a candidate triangle: its entry b
            const uint32_t* cs = L.candSorted + size_t(pt) * L.K;
            uint32_t x = 0, e = L.K;
            while (x < e) {
                const uint32_t mid = (x + e) >> 1;
                if (__ldg(cs + mid) < t) x = mid + 1;
                else e = mid;
            }
            if (x < L.K && __ldg(cs + x) == t) b = j * layerK + l * L.K + __ldg(L.candRank + size_t(pt) * L.K + x);
        }
    }
    p = t + l * m.T;
    float pf = 0.0f;
    if (L.farShare > 0.0f) {
        const float bv = __ldg(m.srcBeta + p) * __ldg(&m.geo[2 * t + 1].z) * m.h;
        const uint32_t nE = F.C * F.slices;
        const float W = float(__ldg(F.rowCdf + size_t(row) * nE + nE - 1));
        const int kImg = imageLevel(ls, int(m.layers), j);
        const float d2 = farDistance2(__ldg(F.cell + cellIdx), S, int(l), kImg, m.h);
        pf = farTerm(farSliceFactor(F.refl, j, int(l) - kImg, m.h, d2), bv, d2,
                     farMeanGain(__ldg(F.gCell + size_t(cellIdx) * m.layers + l), gs,
                                 __ldg(F.gMid + size_t(row) * F.C + cellIdx))) /
             W;
    }
    const float qb = b != 0xffffffffu ? float(__ldg(q + b)) : 0.0f;
    qf = fmaf(L.nearShare, qb, L.farShare * float(Qn) * pf);
    bsel = b;
    return qf > 0.0f;
}

// Persistent ray kernel: every warp repeatedly takes a work item -- itemRays
// consecutive rays of one active sample -- from a global counter, walks them
// (lanes whose ray ends take the next ray of the item, in groups of at least
// REFILL idle lanes so start-point code runs convergent), and writes the
// item's FP64 sums.  No block barrier; per-item partials keep the result
// independent of which warp ran which item.
// POOL: the rows belong to many gain media; the warp copies the view of its
// item's medium into its shared-memory slot (when the medium changes) and
// walks from there, and the number of active rows is read on the device.
// WALK: how the walk obtains each prism's g (WalkMode).
template <int BLOCK, int REFILL, int MINB, bool LOG = false, bool POOL = false, int COLS = kWalkColumns,
          int WALK = kWalkBeta, bool LOCAL = false>
__global__ void __launch_bounds__(BLOCK, MINB) rayKernel(RayLaunch L) {
    __shared__ InstanceView sInst[POOL ? BLOCK / 32 : 1];
    const int lane = threadIdx.x & 31;
    const unsigned laneLt = (1u << lane) - 1u;
    const uint32_t nItems = (POOL ? *L.count : L.nActive) * L.itemsPerRow;
    uint32_t curInst = 0xffffffffu;
    while (true) {
        uint32_t item = 0;
        if (lane == 0) item = atomicAdd(L.itemCounter, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= nItems) break;
        const uint32_t row = L.active[item / L.itemsPerRow];
        const uint32_t k = item % L.itemsPerRow;
        const size_t slot = size_t(row) * kMaxItems + k;
        const unsigned long long Qrow = L.Q[row];
        if (!LOCAL && Qrow == 0ull) {  // no source prism: every ray contributes 0
            if (lane == 0) {
                L.pSum[slot] = 0.0;
                L.pSum2[slot] = 0.0;
                L.pDrop[slot] = 0u;
                L.pCross[slot] = 0ull;
            }
            continue;
        }
        uint32_t sample, nW;
        size_t wBase, oBase;
        if constexpr (POOL) {
            const RowInfo ri = L.rows[row];
            if (ri.inst != curInst) {
                const uint32_t* src = reinterpret_cast<const uint32_t*>(L.inst + ri.inst);
                uint32_t* dst = reinterpret_cast<uint32_t*>(sInst + (threadIdx.x >> 5));
                for (uint32_t w = uint32_t(lane); w < sizeof(InstanceView) / 4; w += 32) dst[w] = __ldg(src + w);
                __syncwarp();
                curInst = ri.inst;
            }
            sample = ri.sample;
            nW = ri.nW;
            wBase = ri.w;
            oBase = ri.w + row;
        } else {
            sample = L.firstSample + row;
            nW = L.nW;
            wBase = size_t(row) * nW;
            oBase = size_t(row) * (nW + 1);
        }
        // per-medium constants: the kernel parameters, or the warp's shared
        // slot, read (volatile) where they are used so that they do not hold
        // registers across the walk
        const volatile InstanceView& iv = sInst[threadIdx.x >> 5];
#define HASE_SEED_LO (POOL ? uint32_t(iv.seedLo) : uint32_t(L.seedLo))
#define HASE_N_LAMBDA (POOL ? uint32_t(iv.nLambda) : uint32_t(L.nLambda))
#define HASE_SPEC (POOL ? (const float2*)iv.spec : L.spec)
        const double Cm = POOL ? double(iv.C) : double(L.C);
        const MeshView& m = POOL ? sInst[threadIdx.x >> 5].m : L.m;
        const GlobalLoader load{m.walk};
        const uint32_t r0 = k * L.itemRays;
        const uint32_t r1 = min(r0 + L.itemRays, L.M);
        const uint32_t* off = L.offsets + oBase;
        const uint32_t* q = L.q + wBase;
        // local proposal without candidate weight (Q = 0): only far rays, their
        // mixture weight taken against Qn = 1
        const unsigned long long Qn = LOCAL && Qrow == 0ull ? 1ull : Qrow;
        const double CQ = Cm * double(Qn);
        const float2 S = __ldg(m.points + sample % m.Np);
        const int ls = int(sample / m.Np);
        // prisms holding the item's mapped rays [r0, rn1): [pb, pb + count - 1)
        // (the local proposal maps its near rays [0, Mnear) only)
        const uint32_t rn1 = LOCAL ? min(r1, L.Mnear) : r1;
        uint32_t bound = 0;
        if (r0 < rn1) {
            if (lane == 0) bound = upperBound(off, nW + 1, r0) - 1u;
            if (lane == 1) bound = upperBound(off, nW + 1, rn1 - 1u) - 1u;
        }
        const uint32_t pb = __shfl_sync(0xffffffffu, bound, 0);
        const uint32_t count = r0 < rn1 ? __shfl_sync(0xffffffffu, bound, 1) - pb + 2u : 0u;

        double sum = 0.0, sum2 = 0.0;
        uint32_t dropped = 0, crossings = 0;
        uint32_t fetch = r0;
        bool active = false;
        Ray ray;
        float wf = 0.0f;
        uint32_t bsel = 0;  // (slice, prism) of the lane's ray, for the contribution log
        while (true) {
            const unsigned idle = __ballot_sync(0xffffffffu, !active);
            const int nIdle = __popc(idle);
            if (fetch >= r1 && nIdle == 32) break;
            if (fetch < r1 && (nIdle >= REFILL || nIdle == 32)) {
                const uint32_t r = fetch + __popc(idle & laneLt);
                if (!active && r < r1) {
                    uint32_t j = 0, p = 0;
                    float qf = 1.0f;
                    bool go = true;
                    if constexpr (LOCAL) {
                        uint32_t bl = 0xffffffffu;
                        go = localSource(L, m, row, sample, S, r, q, off, pb, count, Qrow, Qn, HASE_SEED_LO, j, p,
                                         qf, bl);
                        if (LOG) bsel = bl;
                    } else {
                        const uint32_t b = pb + upperBound(off + pb, count, r) - 1u;
                        if (LOG) bsel = b;
                        // reflection slice by subtraction (at most 4)
                        p = b;
                        while (p >= m.P) {
                            p -= m.P;
                            ++j;
                        }
                        qf = float(__ldg(q + b));
                    }
                    if (go) {
                        const float D2 = startRay(m, r, j, p, sample, S, ls, L.pass, HASE_SEED_LO, L.seedHi,
                                                  __ldg(HASE_SPEC), qf, L.nearField, ray, wf);
                        active = D2 > 0.0f;
                        if (!active) ++dropped;  // start point on the sample point itself
                    }
                }
                fetch += uint32_t(nIdle);
            }
            if (active) {
                const int st = stepRay<COLS, WALK>(m, S.x, S.y, ray, load);
                if (st != kContinue) {
                    crossings += uint32_t(ray.steps) + 1u;
                    if (st == kDone) {
                        finishReflections(m, ray);
                        // the ray's gain in FP32 (FP64 only where exp(G)
                        // nears the FP32 range; the sums stay FP64), averaged
                        // over the spectrum by the beta walks
                        double eg;
                        if constexpr (WALK == kWalkTable)
                            eg = ray.G < 80.0f ? double(expf(ray.G)) : exp(double(ray.G));
                        else
                            eg = rayMeanGain(ray, HASE_SPEC, HASE_N_LAMBDA);
                        const double X = CQ * double(wf) * eg;
                        sum += X;
                        sum2 += X * X;
                        if (LOG && (!LOCAL || bsel != 0xffffffffu)) atomicAdd(L.logBuf + wBase + bsel, float(X));
                    } else {
                        ++dropped;
                    }
                    active = false;
                }
            }
        }
#undef HASE_SEED_LO
#undef HASE_N_LAMBDA
#undef HASE_SPEC
        sum = warpSum(sum);
        sum2 = warpSum(sum2);
        dropped = warpSum(dropped);
        crossings = warpSum(crossings);
        if (lane == 0) {
            L.pSum[slot] = sum;
            L.pSum2[slot] = sum2;
            L.pDrop[slot] = dropped;
            L.pCross[slot] = crossings;
        }
    }
}

// Launch shapes of rayKernel the autotuner chooses from: block size, idle
// lanes that trigger a refill, the occupancy target (blocks per SM the
// register budget is fitted to) and the triangle columns a lane walks per
// step call (32 unless named).  Entry 0 is the default.  Single-medium shapes
// also carry the kernels of the other walk modes.
struct RayVariant {
    void (*kernel)(RayLaunch);
    int block;
    const char* name;
    void (*mono)(RayLaunch);     // the same shape walking the g table (monochromatic single-medium solves), or null
    void (*noClad)(RayLaunch);   // the same shape for a medium without cladding prisms, or null
};
#define HASE_RAY_SHAPE(B, R, M, C, NAME)                                                      \
    {rayKernel<B, R, M, false, false, C>, B, NAME, rayKernel<B, R, M, false, false, C, kWalkTable>, \
     rayKernel<B, R, M, false, false, C, kWalkBetaNoClad>}
const RayVariant kRayVariants[] = {
    HASE_RAY_SHAPE(256, 8, 5, kWalkColumns, "block256_refill8_occ5"),
    HASE_RAY_SHAPE(256, 4, 5, kWalkColumns, "block256_refill4_occ5"),
    HASE_RAY_SHAPE(256, 16, 5, kWalkColumns, "block256_refill16_occ5"),
    HASE_RAY_SHAPE(256, 8, 4, kWalkColumns, "block256_refill8_occ4"),
    HASE_RAY_SHAPE(256, 8, 6, kWalkColumns, "block256_refill8_occ6"),
    HASE_RAY_SHAPE(128, 8, 10, kWalkColumns, "block128_refill8_occ10"),
    HASE_RAY_SHAPE(128, 8, 12, kWalkColumns, "block128_refill8_occ12"),
    HASE_RAY_SHAPE(512, 8, 2, kWalkColumns, "block512_refill8_occ2"),
    HASE_RAY_SHAPE(256, 16, 5, 64, "block256_refill16_occ5_cols64"),
    HASE_RAY_SHAPE(512, 8, 2, 64, "block512_refill8_occ2_cols64"),
};
#undef HASE_RAY_SHAPE
constexpr uint32_t kNumRayVariants = sizeof(kRayVariants) / sizeof(kRayVariants[0]);
static_assert(kNumRayVariants <= 16, "variantBlocks holds 16 launch shapes");
// The same launch shapes for batched media (same order and names): the
// general walk, and the walk for batches without cladding prisms.
#define HASE_POOL_SHAPE(B, R, M, C, NAME) \
    {rayKernel<B, R, M, false, true, C>, B, NAME, nullptr, rayKernel<B, R, M, false, true, C, kWalkBetaNoClad>}
const RayVariant kPoolVariants[] = {
    HASE_POOL_SHAPE(256, 8, 5, kWalkColumns, "block256_refill8_occ5"),
    HASE_POOL_SHAPE(256, 4, 5, kWalkColumns, "block256_refill4_occ5"),
    HASE_POOL_SHAPE(256, 16, 5, kWalkColumns, "block256_refill16_occ5"),
    HASE_POOL_SHAPE(256, 8, 4, kWalkColumns, "block256_refill8_occ4"),
    HASE_POOL_SHAPE(256, 8, 6, kWalkColumns, "block256_refill8_occ6"),
    HASE_POOL_SHAPE(128, 8, 10, kWalkColumns, "block128_refill8_occ10"),
    HASE_POOL_SHAPE(128, 8, 12, kWalkColumns, "block128_refill8_occ12"),
    HASE_POOL_SHAPE(512, 8, 2, kWalkColumns, "block512_refill8_occ2"),
    HASE_POOL_SHAPE(256, 16, 5, 64, "block256_refill16_occ5_cols64"),
    HASE_POOL_SHAPE(512, 8, 2, 64, "block512_refill8_occ2_cols64"),
};
#undef HASE_POOL_SHAPE
static_assert(sizeof(kPoolVariants) == sizeof(kRayVariants), "one batched variant per launch shape");
// Ray kernels of the local proposal: the default's persistent 512-thread,
// 64-column shape in every walk mode, and the contribution-logging kernel.
const RayVariant kLocalVariant{rayKernel<512, 8, 2, false, false, 64, kWalkBeta, true>, 512, "local",
                               rayKernel<512, 8, 2, false, false, 64, kWalkTable, true>,
                               rayKernel<512, 8, 2, false, false, 64, kWalkBetaNoClad, true>};

// ------------------------------------------------ (c)+(d) finalise ----
struct FinalizeLaunch {
    const uint32_t* active;
    uint32_t nActive, items, M;
    int last;                     // no further pass follows
    double threshold;
    const double* pSum;
    const double* pSum2;
    const uint32_t* pDrop;
    const unsigned long long* pCross;
    double* accSum;               // [rows]
    double* accSum2;
    uint32_t* accTotal;
    uint32_t* accDrop;
    unsigned long long* accCross;
    float* phi;                   // [rows]
    double* mse;
    uint32_t* nextActive;
    uint32_t* nextCount;
    const unsigned int* count;    // batched media: the number of active rows (device); warps stride over them
};

__device__ void finalizeRow(const FinalizeLaunch& L, uint32_t row, int lane);

__global__ void __launch_bounds__(128) finalizeKernel(FinalizeLaunch L) {
    const uint32_t n = L.count ? *L.count : L.nActive;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; wid < n; wid += warps)
        finalizeRow(L, L.active[wid], threadIdx.x & 31);
}

__device__ void finalizeRow(const FinalizeLaunch& L, uint32_t row, int lane) {
    double s = 0.0, s2 = 0.0;
    uint32_t d = 0;
    unsigned long long c = 0;
    for (uint32_t k = lane; k < L.items; k += 32) {
        const size_t i = size_t(row) * kMaxItems + k;
        s += L.pSum[i];
        s2 += L.pSum2[i];
        d += L.pDrop[i];
        c += L.pCross[i];
    }
    s = warpSum(s);
    s2 = warpSum(s2);
    d = warpSum(d);
    c = warpSum(c);
    if (lane == 0) {
        const double sum = L.accSum[row] + s, sum2 = L.accSum2[row] + s2;
        const uint32_t N = L.accTotal[row] + L.M;
        L.accSum[row] = sum;
        L.accSum2[row] = sum2;
        L.accTotal[row] = N;
        L.accDrop[row] += d;
        L.accCross[row] += c;
        const double mean = sum / double(N);
        const double rse = mean > 0.0 ? sqrt(fabs(sum2 / double(N) - mean * mean) / double(N)) / mean : 0.0;
        L.phi[row] = float(mean);
        L.mse[row] = rse;
        // Above the threshold: queue for the next pass, or (last pass) just count.
        if (!(rse <= L.threshold)) {
            const uint32_t slot = atomicAdd(L.nextCount, 1u);
            if (!L.last) L.nextActive[slot] = row;
        }
    }
}

__global__ void iotaKernel(uint32_t* a, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
}

// Batched learned solve, after the first pass: the still-active rows whose
// per-ray relative variance (rays x relative error^2) exceeds the limit are
// flagged to restart with the importance weights (counted in *flagged).
__global__ void fallbackMarkKernel(const uint32_t* active, const unsigned int* count, const uint32_t* total,
                                   const double* rse, double limit, uint8_t* flag, unsigned int* flagged) {
    const uint32_t n = *count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t row = active[i];
        const double v = double(total[row]) * rse[row] * rse[row];
        if (!(v <= limit)) {
            flag[row] = 1;
            atomicAdd(flagged, 1u);
        }
    }
}

// Zeroes the accumulators of the flagged active rows.
__global__ void resetFlaggedKernel(const uint32_t* active, const unsigned int* count, const uint8_t* flag,
                                   double* sum, double* sum2, uint32_t* total, uint32_t* drop,
                                   unsigned long long* cross) {
    const uint32_t n = *count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t row = active[i];
        if (!flag[row]) continue;
        sum[row] = 0.0;
        sum2[row] = 0.0;
        total[row] = 0u;
        drop[row] = 0u;
        cross[row] = 0ull;
    }
}

// iota plus the device-held row count of a batched solve's first pass.
__global__ void iotaCountKernel(uint32_t* a, uint32_t n, unsigned int* count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
    if (i == 0) *count = n;
}

// ------------------------------------------------------ diagnostics ----
struct TraceLaunch {
    MeshView m;
    uint32_t n;
    const float* start;
    const uint32_t* tri;
    const uint32_t* level;
    const uint32_t* sample;
    const uint32_t* slice;
    float A, B;
    float* lnGain;
    float* dist;
    uint32_t* dropped;
};

__global__ void traceKernel(TraceLaunch L) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n) return;
    const MeshView& m = L.m;
    const uint32_t sample = L.sample[i];
    const float2 S = __ldg(m.points + sample % m.Np);
    const int ls = int(sample / m.Np);
    const uint32_t j = L.slice[i];
    const int kImg = imageLevel(ls, int(m.layers), j);
    const float zImgOffset = float(kImg) * m.h;
    Ray r;
    const float D2 = initRay(r, L.tri[i], int(L.level[i]), L.start[3 * i] - S.x, L.start[3 * i + 1] - S.y,
                             L.start[3 * i + 2] - zImgOffset, kImg, j, L.A, L.B, m);
    GlobalLoader load{m.walk};
    int st;
    do {
        st = stepRay(m, S.x, S.y, r, load);
    } while (st == kContinue);
    if (st == kDone) finishReflections(m, r);
    L.lnGain[i] = r.G;
    L.dist[i] = sqrtf(D2);
    L.dropped[i] = st == kDone ? 0u : 1u;
}

__global__ void philoxKernel(uint32_t n, const uint32_t* ctr, uint32_t k0, uint32_t k1, uint32_t* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Philox4 r = philox4x32_10(ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3], k0, k1);
    out[4 * i] = r.x;
    out[4 * i + 1] = r.y;
    out[4 * i + 2] = r.z;
    out[4 * i + 3] = r.w;
}

// ---------------------------------------------------------- L2 probe ----
// Reads an L2-resident buffer `reps` times with 16-byte loads from every SM;
// the bench uses it as the measured L2 read bandwidth of the gather roofline.
__global__ void __launch_bounds__(512) l2ProbeKernel(const float4* __restrict__ buf, size_t n, uint32_t reps,
                                                     float* sink) {
    float acc = 0.0f;
    const size_t stride = size_t(gridDim.x) * blockDim.x;
    for (uint32_t r = 0; r < reps; ++r)
        for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += stride) {
            const float4 v = __ldcg(buf + i);
            acc += v.x + v.y + v.z + v.w;
        }
    if (acc == 1234.5f) *sink = acc;  // keeps the loads; never true for a zeroed buffer
}

// L1 and shared-memory read bandwidth probes: every block reads the same
// 32 KB (which stays resident in each SM's L1, or in the block's shared
// memory) `reps` times with 16-byte loads.  The loads are volatile inline
// PTX, so none is hoisted out of the repeat loop.
constexpr uint32_t kProbeVec = 2048;  // float4 elements: 32 KB
__global__ void __launch_bounds__(1024) l1ProbeKernel(const float4* __restrict__ buf, uint32_t reps, float* sink) {
    float a = 0.0f, b = 0.0f, c = 0.0f, d = 0.0f;
    for (uint32_t r = 0; r < reps; ++r)
        for (uint32_t i = threadIdx.x; i < kProbeVec; i += blockDim.x) {
            float x, y, z, w;
            asm volatile("ld.global.nc.v4.f32 {%0, %1, %2, %3}, [%4];"
                         : "=f"(x), "=f"(y), "=f"(z), "=f"(w)
                         : "l"(buf + i));
            a += x;
            b += y;
            c += z;
            d += w;
        }
    if (a + b + c + d == 1234.5f) *sink = a;  // never true for a zeroed buffer
}

__global__ void __launch_bounds__(1024) smemProbeKernel(uint32_t reps, float* sink) {
    __shared__ float4 buf[kProbeVec];
    for (uint32_t i = threadIdx.x; i < kProbeVec; i += blockDim.x) buf[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    __syncthreads();
    float a = 0.0f, b = 0.0f, c = 0.0f, d = 0.0f;
    for (uint32_t r = 0; r < reps; ++r)
        for (uint32_t i = threadIdx.x; i < kProbeVec; i += blockDim.x) {
            float x, y, z, w;
            const uint32_t addr = uint32_t(__cvta_generic_to_shared(buf + i));
            asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                         : "=f"(x), "=f"(y), "=f"(z), "=f"(w)
                         : "r"(addr));
            a += x;
            b += y;
            c += z;
            d += w;
        }
    if (a + b + c + d == 1234.5f) *sink = a;
}

// ------------------------------------------- allocation-free estimate ----
// Scratch of hase_estimate_sample_noalloc: a file-scope device array, so that
// entry point never allocates.  Every GPU that loads this library holds it
// (about 4.2 MiB) until the process exits; all calls on one GPU share it.
constexpr uint32_t kNoAllocMaxPrismSlices = 1u << 19;  // reflection slices x prisms per sample
constexpr size_t kNoAllocQ = 0;                                              // u32 [max]
constexpr size_t kNoAllocOffsets = kNoAllocQ + 4ull * kNoAllocMaxPrismSlices;  // u32 [max + 1]
constexpr size_t kNoAllocSmall = kNoAllocOffsets + 4ull * kNoAllocMaxPrismSlices + 256;
// small block: Q u64, active u32, itemCounter u32, nextActive u32, nextCount u32,
// accSum f64, accSum2 f64, accTotal u32, accDrop u32, accCross u64, phi f32, mse f64
constexpr size_t kNoAllocPartials = kNoAllocSmall + 256;  // f64, f64, u32, u64 [kMaxItems] each
constexpr size_t kNoAllocBytes = kNoAllocPartials + size_t(kMaxItems) * (8 + 8 + 4 + 8);

static __device__ __align__(256) unsigned char g_noAllocScratch[kNoAllocBytes];

__global__ void noAllocEmitKernel(const float* phi, const double* mse, const uint32_t* total, const uint32_t* drop,
                                  double* out) {
    out[0] = double(*phi);
    out[1] = *mse;
    out[2] = double(*total);
    out[3] = double(*drop);
}

// ------------------------------------------------- learned proposal ----
// Features of a (sample, slice, prism) pair (include/hase_b200_proposal.h)
// and the defensive-mixture weights that replace the importance weights.
struct ProposalView {
    MeshView m;
    const float* grid;      // [layers][gy][gx] mean gain coefficient per cell (1/cm)
    uint32_t gx, gy;
    float x0, y0, invCell;  // grid origin and 1 / cell size
    float lnRb, lnRt;       // mean ln reflectivity of the bottom and top surfaces
    float R, H;             // mesh radius and height
    float invR, invH, invTwoH, invh;  // 1/R, 1/H, 1/(2H), 1/(level spacing)
    float lnVref;           // ln(mean prism volume / R^2)
    float lnSigmaRatio;     // ln(sigma_e / sigma_a) of the averaged spectrum
    uint32_t firstSample, nW;
    // local proposal: pair jp is candidate entry j (layers K) + l K + k of the
    // sample's point (cand null: jp = j P + prism)
    const uint32_t* cand;
    uint32_t K, divKm, divKs;
};

__device__ __forceinline__ float sliceLnReflect(const ProposalView& V, uint32_t j) {
    return j == 0 ? 0.0f : j == 1 ? V.lnRb : j == 2 ? V.lnRt : V.lnRb + V.lnRt;
}

// Returns the prior beta V R_j / d^2 (0 without a source) and fills f.
__device__ __forceinline__ float pairFeatures(const ProposalView& V, uint32_t sample, uint32_t jp, float (&f)[kFeat]) {
    const MeshView& m = V.m;
    // (slice, prism) and (triangle, layer), sample point and level: no
    // integer divisions (slices by subtraction, the rest by multiply-shift)
    const uint32_t lsU = sampleLevel(m, sample);
    const uint32_t pt = sample - lsU * m.Np;
    uint32_t j = 0, p = jp, l, t;
    if (V.cand) {
        const uint32_t layerK = m.layers * V.K;
        while (p >= layerK) {
            p -= layerK;
            ++j;
        }
        l = uint32_t((uint64_t(p) * V.divKm) >> V.divKs);
        t = __ldg(V.cand + size_t(pt) * V.K + (p - l * V.K));
        p = t + l * m.T;
    } else {
        while (p >= m.P) {
            p -= m.P;
            ++j;
        }
        l = prismLayer(m, p);
        t = p - l * m.T;
    }
    const float2 S = __ldg(m.points + pt);
    const int ls = int(lsU);
    const float zs = float(ls) * m.h;
    const float zi = float(imageLevel(ls, int(m.layers), j)) * m.h;
    const float2 c = __ldg(m.centroid + t);
    const float zc = (float(l) + 0.5f) * m.h;
    const float dx = c.x - S.x, dy = c.y - S.y, dz = zc - zi;
    const float d = sqrtf(dx * dx + dy * dy + dz * dz);
    const float beta = __ldg(m.srcBeta + p);
    const float vol = __ldg(m.geo + 2 * t + 1).z * m.h;
    // straight-line ln gain estimated on the coarse grid, 8 points, z folded
    float lng = 0.0f;
    const float twoH = 2.0f * V.H;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float a = (float(k) + 0.5f) * 0.125f;
        const float x = S.x + a * dx, y = S.y + a * dy;
        // fold the unfolded height into [0, H]: period 2H, mirrored halves
        float z = zi + a * dz;
        z -= twoH * floorf(z * V.invTwoH);
        if (z > V.H) z = twoH - z;
        const int ly = min(max(int(z * V.invh), 0), int(m.layers) - 1);
        const int ix = min(max(int((x - V.x0) * V.invCell), 0), int(V.gx) - 1);
        const int iy = min(max(int((y - V.y0) * V.invCell), 0), int(V.gy) - 1);
        lng += __ldg(V.grid + (size_t(ly) * V.gy + iy) * V.gx + ix);
    }
    const float lnR = sliceLnReflect(V, j);
    lng = lng * 0.125f * d + lnR;
    f[0] = S.x * V.invR;
    f[1] = S.y * V.invR;
    f[2] = zs * V.invH;
    f[3] = dx * V.invR;
    f[4] = dy * V.invR;
    f[5] = dz * V.invH;
    f[6] = logf(d * V.invR);
    f[7] = beta;
    f[8] = lng;
    f[9] = beta > 0.0f ? logf(beta * vol / (d * d)) - V.lnVref : 0.0f;
    f[10] = float(j) * 0.25f;
    f[11] = V.lnSigmaRatio;
    return beta > 0.0f ? beta * vol * __expf(lnR) / (d * d) : 0.0f;
}

struct ProposalLaunch {
    ProposalView V;
    const uint4* wimg;
    const float* vec;
    float* out;             // [rows][nW]: logits
    float* prior;           // [rows][nW]: beta V R_j / d^2 (0 without a source)
    float* features;        // [rows][nW][kFeat] (featureKernel) or null
    uint32_t rows;          // sample rows from V.firstSample
    int* error;
};

// Network logits of every (slice, prism) of `rows` sample rows (tensor cores).
__global__ void __launch_bounds__(kTile, kMlpBlocksPerSM) proposalKernel(const ProposalLaunch P) {
    extern __shared__ uint8_t dynSmem[];
    Tile T;
    tileBegin<SmemMap>(T, dynSmem, P.wimg, P.vec);
    const uint64_t total = uint64_t(P.rows) * P.V.nW;
    const uint64_t tiles = (total + kTile - 1) / kTile;
    // (row, column) of this thread's pair, advanced by the grid stride without
    // a division per tile
    const uint64_t gr0 = uint64_t(blockIdx.x) * kTile + threadIdx.x;
    const uint64_t stride = uint64_t(gridDim.x) * kTile;
    uint32_t row = uint32_t(gr0 / P.V.nW), col = uint32_t(gr0 % P.V.nW);
    const uint32_t dRow = uint32_t(stride / P.V.nW), dCol = uint32_t(stride % P.V.nW);
    for (uint64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint64_t gr = tile * kTile + threadIdx.x;
        float f[kFeat];
        if (gr < total) {
            P.prior[gr] = pairFeatures(P.V, P.V.firstSample + row, col, f);
        } else {
#pragma unroll
            for (int k = 0; k < kFeat; ++k) f[k] = 0.0f;
        }
        storeFeatures(T, SmemMap::a0, f);
        const float logit = mlpTile<true>(T);
        if (gr < total) P.out[gr] = logit;
        col += dCol;
        row += dRow;
        if (col >= P.V.nW) {
            col -= P.V.nW;
            ++row;
        }
        if (!__syncthreads_and(T.ok)) break;
    }
    tileEnd<SmemMap>(T, P.error);
}

// Feature rows only (training sets): one thread per pair.
__global__ void featureKernel(const ProposalLaunch P) {
    const uint64_t gr = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (gr >= uint64_t(P.rows) * P.V.nW) return;
    float f[kFeat];
    pairFeatures(P.V, P.V.firstSample + uint32_t(gr / P.V.nW), uint32_t(gr % P.V.nW), f);
#pragma unroll
    for (int k = 0; k < kFeat; ++k) P.features[gr * kFeat + k] = f[k];
}

// The coarse-grid proposal (hase_context_set_grid_proposal): the importance
// function beta V R / d^2 e^G of a (slice, prism) pair with the straight-line
// gain G taken from the coarse gain grid (the 8-point estimate of the
// features, pairFeatures) instead of a walk, and the slice's reflection
// factor R taken per bounce from the pair's own direction: 1 beyond the
// critical angle of the surface, the surface's mean reflectivity otherwise.
// ln w; -inf without a source.
//
// Only what the weight uses is computed.  A thread takes one column (prism,
// or candidate entry l K + k) of a sample row and every reflection slice of
// it: the sample point, the prism's centroid, beta V and the in-plane cells
// of the 8 gain points do not depend on the slice, so they are found once;
// per slice only the folded height of the 8 points, d^2 and the bounce
// factor remain.  Rows come from the grid's y dimension (no 64-bit division
// per pair).

// floor(v) of 0 <= v < 2^22 as an integer, on the FP32 pipe: adding 1.5 2^23
// rounded toward -inf leaves floor(v) in the low mantissa bits.
__device__ __forceinline__ int floorSmall(float v) {
    return __float_as_int(__fadd_rd(v, 12582912.0f)) - 0x4B400000;
}

// min(max(int(v), 0), hi) for finite v (the cell index of pairFeatures).
__device__ __forceinline__ int clampedCell(float v, int hi) {
    return floorSmall(fminf(fmaxf(v, 0.0f), float(hi)));
}

// ln w of every pair of `rows` sample rows from the coarse grid (P.out).
// Launch: x covers the columns of one slice (P.V.cand ? layers K : P),
// y the rows (strided past 65535).
__global__ void __launch_bounds__(256) gridWeightKernel(const ProposalLaunch P) {
    const ProposalView& V = P.V;
    const MeshView& m = V.m;
    const uint32_t width = V.cand ? m.layers * V.K : m.P;
    const uint32_t col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= width) return;
    const uint32_t slices = V.nW / width;
    // the column's layer and its triangle (full rows) or candidate rank
    uint32_t l, k;
    if (V.cand) {
        l = uint32_t((uint64_t(col) * V.divKm) >> V.divKs);
        k = col - l * V.K;
    } else {
        l = prismLayer(m, col);
        k = col - l * m.T;
    }
    const float zc = (float(l) + 0.5f) * m.h;
    const float twoH = 2.0f * V.H;
    const uint32_t gxy = V.gx * V.gy;
    for (uint32_t row = blockIdx.y; row < P.rows; row += gridDim.y) {
        const uint32_t sample = V.firstSample + row;
        const uint32_t lsU = sampleLevel(m, sample);
        const uint32_t pt = sample - lsU * m.Np;
        const uint32_t t = V.cand ? __ldg(V.cand + size_t(pt) * V.K + k) : k;
        const uint32_t p = t + l * m.T;
        float* out = P.out + size_t(row) * V.nW + col;
        const float beta = __ldg(m.srcBeta + p);
        if (!(beta > 0.0f)) {
            for (uint32_t j = 0; j < slices; ++j) out[size_t(j) * width] = -INFINITY;
            continue;
        }
        const float2 S = __ldg(m.points + pt);
        const float2 c = __ldg(m.centroid + t);
        const float dx = c.x - S.x, dy = c.y - S.y;
        const float r2 = dx * dx + dy * dy;
        const float lnBV = __logf(beta * (__ldg(m.geo + 2 * t + 1).z * m.h));
        // in-plane cell of each gain point: the same for every slice
        uint32_t cellXY[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const float a = (float(q) + 0.5f) * 0.125f;
            const float x = S.x + a * dx, y = S.y + a * dy;
            const int ix = clampedCell((x - V.x0) * V.invCell, int(V.gx) - 1);
            const int iy = clampedCell((y - V.y0) * V.invCell, int(V.gy) - 1);
            cellXY[q] = uint32_t(iy) * V.gx + uint32_t(ix);
        }
        const int ls = int(lsU);
        for (uint32_t j = 0; j < slices; ++j) {
            const float zi = float(imageLevel(ls, int(m.layers), j)) * m.h;
            const float dz = zc - zi;
            const float d2 = fmaf(dz, dz, r2);
            float lng = 0.0f;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const float a = (float(q) + 0.5f) * 0.125f;
                // fold the unfolded height into [0, H]: period 2H, mirrored halves
                float z = zi + a * dz;
                const float fl = __fadd_rd(z * V.invTwoH, 12582912.0f) - 12582912.0f;  // floor, |.| < 2^22
                z -= twoH * fl;
                if (z > V.H) z = twoH - z;
                const uint32_t ly = uint32_t(clampedCell(z * V.invh, int(m.layers) - 1));
                lng += __ldg(V.grid + ly * gxy + cellXY[q]);
            }
            float lnR = 0.0f;
            if (j > 0) {
                const float dz2 = dz * dz;
                const float lb = dz2 <= m.tirCos2[0] * d2 ? 0.0f : V.lnRb;
                const float lt = dz2 <= m.tirCos2[1] * d2 ? 0.0f : V.lnRt;
                lnR = j == 1 ? lb : (j == 2 ? lt : lb + lt);
            }
            const float d = d2 * rsqrtf(d2);
            out[size_t(j) * width] = fmaf(lng * 0.125f, d, lnBV - __logf(d2) + lnR);
        }
    }
}

// Launches gridWeightKernel over `gl.rows` rows of gl.V.nW pairs.
static cudaError_t launchGridWeights(const ProposalLaunch& gl, cudaStream_t s) {
    const uint32_t width = gl.V.cand ? gl.V.m.layers * gl.V.K : gl.V.m.P;
    if (width == 0 || gl.rows == 0) return cudaSuccess;
    const dim3 grid((width + 255) / 256, std::min<uint32_t>(gl.rows, 65535u));
    gridWeightKernel<<<grid, 256, 0, s>>>(gl);
    return cudaGetLastError();
}

template <bool MAX>
__device__ __forceinline__ float blockReduce1024(float v, float* red) {
    for (int o = 16; o > 0; o >>= 1) {
        const float w = __shfl_xor_sync(0xffffffffu, v, o);
        v = MAX ? fmaxf(v, w) : v + w;
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    v = red[0];
    for (int k = 1; k < int(blockDim.x >> 5); ++k) v = MAX ? fmaxf(v, red[k]) : v + red[k];
    return v;
}

// One block per sample row: lnw = ln((1 - alpha) softmax(logits) + alpha
// prior / sum prior) over the pairs with a source (prior > 0), -inf elsewhere.
__global__ void __launch_bounds__(1024) mixtureKernel(uint32_t nW, float* lnw, const float* priorBuf, float alpha) {
    __shared__ float red[32];
    const uint32_t row = blockIdx.x;
    float* w = lnw + size_t(row) * nW;
    const float* pr = priorBuf + size_t(row) * nW;
    float mx = -INFINITY, ps = 0.0f;
    for (uint32_t jp = threadIdx.x; jp < nW; jp += blockDim.x) {
        const float prior = pr[jp];
        if (prior > 0.0f) {
            mx = fmaxf(mx, w[jp]);
            ps += prior;
        }
    }
    mx = blockReduce1024<true>(mx, red);
    ps = blockReduce1024<false>(ps, red);
    float se = 0.0f;
    for (uint32_t jp = threadIdx.x; jp < nW; jp += blockDim.x)
        if (pr[jp] > 0.0f) se += __expf(w[jp] - mx);
    se = blockReduce1024<false>(se, red);
    const float a = ps > 0.0f ? alpha / ps : 0.0f, b = se > 0.0f ? (1.0f - alpha) / se : 0.0f;
    for (uint32_t jp = threadIdx.x; jp < nW; jp += blockDim.x) {
        const float prior = pr[jp];
        const float q = prior > 0.0f ? b * __expf(w[jp] - mx) + a * prior : 0.0f;
        w[jp] = q > 0.0f ? logf(q) : -INFINITY;
    }
}

// Zeroes the accumulators of the listed rows (samples restarted with the
// exact importance weights).
__global__ void resetRowsKernel(const uint32_t* rows, uint32_t n, double* sum, double* sum2, uint32_t* total,
                                uint32_t* drop, unsigned long long* cross) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t r = rows[i];
    sum[r] = 0.0;
    sum2[r] = 0.0;
    total[r] = 0u;
    drop[r] = 0u;
    cross[r] = 0ull;
}

// ------------------------------------------------ time stepping ----
// Rate equations of the excited fraction per prism (hase_simulate).
struct PumpLaunch {
    const float2* centroid;       // [T]
    const double* beta;           // [P] stage beta
    const uint8_t* clad;          // [P] 1 = cladding prism, or null
    double* rate;                 // [P] out: d beta / dt from the pump
    double* absorbed;             // [1] absorbed photon flux x area (first stage diagnostics), or null
    const float* area;            // [T]
    uint32_t T, layers;
    double h, nTot, sA, sE, cladAbs;
    double flux0, radius, expo, cx, cy;  // peak photon flux (1/(cm^2 s)), profile
    int retro;
};

// One thread per triangle column: Beer-Lambert up the column (and back down
// with retro-reflection); each layer's absorbed photons / (N_tot h).
__global__ void pumpColumnKernel(const PumpLaunch L) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= L.T) return;
    const float2 c = L.centroid[t];
    const double r = sqrt(double(c.x - L.cx) * double(c.x - L.cx) + double(c.y - L.cy) * double(c.y - L.cy));
    double phi = L.flux0 * exp(-pow(r / L.radius, L.expo));
    const double phi0 = phi;
    for (int pass = 0; pass < (L.retro ? 2 : 1); ++pass) {
        for (uint32_t k = 0; k < L.layers; ++k) {
            const uint32_t l = pass == 0 ? k : L.layers - 1 - k;
            const size_t p = t + size_t(l) * L.T;
            const bool cl = L.clad && L.clad[p];
            const double g = cl ? -L.cladAbs : L.nTot * (L.beta[p] * (L.sA + L.sE) - L.sA);
            const double out = phi * exp(g * L.h);
            if (!cl) L.rate[p] += (phi - out) / (L.nTot * L.h);
            phi = out;
        }
    }
    if (L.absorbed) atomicAdd(L.absorbed, (phi0 - phi) * double(L.area[t]));
}

// Mean phi-ASE of each prism's six vertices (levels l and l + 1).
__global__ void phiPrismKernel(const int4* verts, const float* phiSample, float* phiPrism, uint32_t T,
                               uint32_t layers, uint32_t Np) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= T * layers) return;
    const uint32_t t = p % T, l = p / T;
    const int4 v = verts[t];
    const float* a = phiSample + size_t(l) * Np;
    const float* b = a + Np;
    phiPrism[p] = (a[v.x] + a[v.y] + a[v.z] + b[v.x] + b[v.y] + b[v.z]) * (1.0f / 6.0f);
}

// Time integrators of hase_simulate (include/core/timeSteppedSimulation.hpp:321-415).
enum TimeIntegrator : uint32_t {
    kFrozenRk4 = 0,      // frozen-phi-ase-runge-kutta-4: phi-ASE solved at the step start only
    kExplicitEuler = 1,  // explicit-euler
    kHeun = 2,           // heun: phi-ASE re-solved at the predictor
    kMidpoint = 3,       // midpoint: phi-ASE re-solved at the midpoint
    kRk4 = 4,            // runge-kutta-4: phi-ASE re-solved at every stage
    kImplicitEuler = 5,  // implicit-euler: fixed-point iterations, phi-ASE re-solved on each
    kExpEuler = 6,       // exponential-euler
    kNumIntegrators = 7,
};

// Derivative of beta at state b (include/kernels/derivativeComposition.hpp:27-63):
// k = pump - [b (sE + sA) - sA] Phi - b / tau, 0 in cladding prisms.
__global__ void rateDerivativeKernel(const double* b, const double* pumpRate, const float* phiPrism,
                                     const uint8_t* clad, double* k, uint32_t P, double sA, double sE, double tau) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    double v = 0.0;
    if (!(clad && clad[p])) {
        const double bp = b[p];
        v = pumpRate[p] - (bp * (sE + sA) - sA) * double(phiPrism ? phiPrism[p] : 0.0f) - bp / tau;
    }
    k[p] = v;
}

// out = base + a k (a stage state, not clipped; AddScaled).
__global__ void rateAxpyKernel(const double* base, const double* k, double a, double* out, uint32_t P) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < P) out[p] = base[p] + a * k[p];
}

// The step's update from its stage derivatives k[0 .. 3] ([4][P]) in the
// reference's forms (AddScaled, CombineHeun, CombineRungeKutta4), clipped to
// [0, 1] (ClipBeta): include/kernels/timeIntegrationUpdateKernels.hpp:21-105.
__global__ void rateCombineKernel(const double* base, const double* k, uint32_t mode, double dt, double* out,
                                  uint32_t P) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    const double* k1 = k;
    const double* k2 = k + P;
    const double* k3 = k + 2 * size_t(P);
    const double* k4 = k + 3 * size_t(P);
    double v;
    switch (mode) {
        case kHeun: v = base[p] + 0.5 * dt * (k1[p] + k2[p]); break;
        case kMidpoint: v = base[p] + dt * k2[p]; break;
        case kFrozenRk4:
        case kRk4: v = base[p] + (dt / 6.0) * (k1[p] + 2.0 * k2[p] + 2.0 * k3[p] + k4[p]); break;
        default: v = base[p] + dt * k1[p]; break;  // explicit and implicit Euler
    }
    out[p] = fmin(1.0, fmax(0.0, v));
}

// Exponential Euler (ExponentialEulerUpdate, include/kernels/timeIntegrationUpdateKernels.hpp:67-90):
// out = tau (pump - ASE term) (1 - e^{-dt/tau}) + b e^{-dt/tau}, the pump and
// ASE terms 0 in cladding prisms, clipped to [0, 1].
__global__ void rateExpEulerKernel(const double* b, const double* pumpRate, const float* phiPrism,
                                   const uint8_t* clad, double* out, uint32_t P, double sA, double sE, double tau,
                                   double dt) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    const double decay = exp(-dt / tau);
    const double bp = b[p];
    double source = 0.0;
    if (!(clad && clad[p])) source = pumpRate[p] - (bp * (sE + sA) - sA) * double(phiPrism ? phiPrism[p] : 0.0f);
    out[p] = fmin(1.0, fmax(0.0, tau * source * (1.0 - decay) + bp * decay));
}

// The context's walk / source beta from the FP64 state (NaN marks cladding in the walk table).
__global__ void betaToTablesKernel(const double* beta, const uint8_t* clad, float* gainBeta, float* srcBeta,
                                   uint32_t P) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    const float b = float(beta[p]);
    srcBeta[p] = b;
    gainBeta[p] = (clad && clad[p]) ? __int_as_float(0x7fc00000) : b;
}

// Gain coefficient of every prism for one (A, B): g = beta A - B
// (-claddingAbsorption in cladding), evaluated exactly as the walks evaluate
// it, so that a walk can read g where it would read beta.  A solve builds it
// for its spectrally averaged (A, B): the importance walks use those, and so
// does the ray walk of a monochromatic solve (the mean of one pair is that pair).
__global__ void gainTableKernel(const float* gainBeta, float A, float B, float cladAbs, uint32_t P, float* g) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    const float b = gainBeta[p];
    g[p] = (b == b) ? fmaf(b, A, -B) : -cladAbs;
}

// -------------------------------------------------------- host side ----
// Multiplier and shift with floor(n / d) = (n * mul) >> shift for every
// n < 2^31 and 1 <= d < 2^32 (Granlund and Montgomery, "Division by invariant
// integers using multiplication", PLDI 1994, theorem 4.2 with N = 31):
// l = ceil(log2 d), mul = ceil(2^(31 + l) / d) (< 2^32), shift = 31 + l.
void invariantDivisor(uint32_t d, uint32_t& mul, uint32_t& shift) {
    uint32_t l = 0;
    while ((uint64_t(1) << l) < d) ++l;
    shift = 31 + l;
    mul = uint32_t(((uint64_t(1) << shift) + d - 1) / d);
}

struct HostTables {
    std::vector<int4> verts;
    std::vector<float4> tri, walk, geo;
    std::vector<float2> centroid, points;
};

hase_status buildHostTables(const hase_mesh_desc* d, HostTables& h, double& extent) {
    const uint32_t T = d->numberOfTriangles, Np = d->numberOfPoints;
    h.tri.assign(3 * size_t(T), make_float4(0, 0, 0, 0));
    h.geo.assign(2 * size_t(T), make_float4(0, 0, 0, 0));
    h.centroid.resize(T);
    h.points.resize(Np);
    h.verts.resize(T);
    extent = 0.0;
    for (uint32_t i = 0; i < Np; ++i) {
        h.points[i] = make_float2(float(d->points[2 * i]), float(d->points[2 * i + 1]));
        extent = std::max(extent, std::max(std::fabs(d->points[2 * i]), std::fabs(d->points[2 * i + 1])));
    }
    std::vector<int32_t> nbr(3 * size_t(T), -1);
    std::unordered_map<uint64_t, uint32_t> open;  // edge key -> 3*t + e
    open.reserve(3 * size_t(T));
    for (uint32_t t = 0; t < T; ++t) {
        const uint32_t* v = d->triangles + 3 * size_t(t);
        for (int e = 0; e < 3; ++e)
            if (v[e] >= Np) return fail(HASE_INVALID_ARGUMENT, "triangle %u references point %u >= %u", t, v[e], Np);
        const double x0 = d->points[2 * v[0]], y0 = d->points[2 * v[0] + 1];
        const double x1 = d->points[2 * v[1]], y1 = d->points[2 * v[1] + 1];
        const double x2 = d->points[2 * v[2]], y2 = d->points[2 * v[2] + 1];
        const double cross = (x1 - x0) * (y2 - y0) - (y1 - y0) * (x2 - x0);
        if (!(std::fabs(cross) > 0.0)) return fail(HASE_INVALID_ARGUMENT, "triangle %u is degenerate", t);
        const double orient = cross > 0.0 ? 1.0 : -1.0;
        double nx[3], ny[3], c[3];
        for (int e = 0; e < 3; ++e) {
            const uint32_t a = v[e], b = v[(e + 1) % 3];
            const double ex = d->points[2 * b] - d->points[2 * a], ey = d->points[2 * b + 1] - d->points[2 * a + 1];
            const double inv = 1.0 / std::sqrt(ex * ex + ey * ey);
            nx[e] = orient * ey * inv;
            ny[e] = -orient * ex * inv;
            c[e] = nx[e] * d->points[2 * a] + ny[e] * d->points[2 * a + 1];
            const uint64_t key = (uint64_t(std::min(a, b)) << 32) | std::max(a, b);
            auto it = open.find(key);
            if (it == open.end()) {
                open.emplace(key, 3 * t + e);
            } else {
                const uint32_t other = it->second;
                if (nbr[other] != -1) return fail(HASE_INVALID_ARGUMENT, "edge shared by more than two triangles");
                nbr[3 * t + e] = int32_t(other);
                nbr[other] = int32_t(3 * t + e);
                open.erase(it);
            }
        }
        h.tri[3 * t + 0] = make_float4(float(nx[0]), float(ny[0]), float(c[0]), float(nx[1]));
        h.tri[3 * t + 1] = make_float4(float(ny[1]), float(c[1]), float(nx[2]), float(ny[2]));
        h.tri[3 * t + 2].x = float(c[2]);
        h.geo[2 * t] = make_float4(float(x0), float(y0), float(x1 - x0), float(y1 - y0));
        h.geo[2 * t + 1] = make_float4(float(x2 - x0), float(y2 - y0), float(0.5 * std::fabs(cross)), 0.0f);
        h.centroid[t] = make_float2(float((x0 + x1 + x2) / 3.0), float((y0 + y1 + y2) / 3.0));
        h.verts[t] = make_int4(int(v[0]), int(v[1]), int(v[2]), 0);
    }
    for (uint32_t t = 0; t < T; ++t) {
        int32_t w[3];
        for (int e = 0; e < 3; ++e) {
            const int32_t o = nbr[3 * t + e];
            w[e] = o < 0 ? -1 : int32_t((uint32_t(o / 3) << 2) | uint32_t(o % 3));
        }
        float* rec = &h.tri[3 * t + 2].y;
        std::memcpy(rec, w, sizeof(w));
    }
    // the walks' copy: a boundary edge's normal is NaN, so its dd > 0 test fails
    // and the walks need no separate boundary test
    h.walk = h.tri;
    const float nan = std::numeric_limits<float>::quiet_NaN();
    for (uint32_t t = 0; t < T; ++t) {
        float* r = &h.walk[3 * size_t(t)].x;  // nx0 ny0 c0 nx1 | ny1 c1 nx2 ny2 | c2 nb0 nb1 nb2
        static const int kNx[3] = {0, 3, 6}, kNy[3] = {1, 4, 7};
        for (int e = 0; e < 3; ++e) {
            int32_t nb;
            std::memcpy(&nb, r + 9 + e, sizeof(nb));
            if (nb < 0) r[kNx[e]] = r[kNy[e]] = nan;
        }
    }
    return HASE_OK;
}

// The far prior's tables of the current beta: per (layer, cell) the cell's
// beta V prefix over its triangles (cellTris order) and its total.  One
// thread per (layer, cell).
__global__ void farCellKernel(const uint32_t* cellStart, const uint32_t* cellTris, uint32_t C, const float* srcBeta,
                              const float4* geo, uint32_t T, uint32_t layers, float h, float* cellMass,
                              float* triPrefix) {
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= C * layers) return;
    const uint32_t l = idx / C, c = idx - l * C;
    const uint32_t s0 = cellStart[c], s1 = cellStart[c + 1];
    float run = 0.0f;
    for (uint32_t i = s0; i < s1; ++i) {
        const uint32_t t = cellTris[i];
        run += srcBeta[size_t(l) * T + t] * geo[2 * t + 1].z * h;
        triPrefix[size_t(l) * T + i] = run;
    }
    cellMass[size_t(c) * layers + l] = run;
}

struct FarRowLaunch {
    const float4* cell;
    const float* cellMass;
    const float* gCell;
    const float* gTab;
    const uint32_t* cand;
    uint32_t C, slices, layers, Np, firstSample, K, T;
    const float2* points;
    float h;
    FarSlices refl;
    double* rowCdf;  // [rows][C][slices]
    float* gMid;     // [rows][C]
    // the layer-averaged coarse gain grid ([gy][gx], origin, 1 / cell size)
    const float* colGrid;
    uint32_t gx, gy;
    float x0, y0, invCell;
};

// The layer average of the coarse gain grid: one thread per (x, y) cell.
__global__ void farColumnKernel(const float* grid, uint32_t cells, uint32_t layers, float* colGrid) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= cells) return;
    float sum = 0.0f;
    for (uint32_t l = 0; l < layers; ++l) sum += grid[size_t(l) * cells + k];
    colGrid[k] = sum / float(layers);
}

// g_mid: the mean of the layer-averaged gain grid at the points a = 1/7 ..
// 6/7 of the 2-D segment from the sample point S to the cell centre.
__device__ __forceinline__ float farMidGain(const FarRowLaunch& L, float2 S, float cx, float cy) {
    const float dx = cx - S.x, dy = cy - S.y;
    float sum = 0.0f;
#pragma unroll
    for (int k = 1; k <= 6; ++k) {
        const float a = float(k) * (1.0f / 7.0f);
        const int ix = clampedCell((S.x + a * dx - L.x0) * L.invCell, int(L.gx) - 1);
        const int iy = clampedCell((S.y + a * dy - L.y0) * L.invCell, int(L.gy) - 1);
        sum += __ldg(L.colGrid + uint32_t(iy) * L.gx + uint32_t(ix));
    }
    return sum * (1.0f / 6.0f);
}

// The far prior's mean g of every (cell, layer) for this solve's gain table.
__global__ void farGainKernel(const uint32_t* cellStart, const uint32_t* cellTris, uint32_t C, const float* gTab,
                              uint32_t T, uint32_t layers, float* gCell) {
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= C * layers) return;
    const uint32_t l = idx / C, c = idx - l * C;
    const uint32_t s0 = cellStart[c], s1 = cellStart[c + 1];
    float sum = 0.0f;
    for (uint32_t i = s0; i < s1; ++i) sum += gTab[size_t(l) * T + cellTris[i]];
    gCell[size_t(c) * layers + l] = sum / float(s1 - s0);
}

// Per sample row of a chunk: the inclusive FP64 prefix over (cell, slice)
// pairs of the far prior's weights w_cj = sum_l term_clj (FP32, layers in
// order, empty layers skipped: the terms localSource's layer scan adds).  One block per row, 256 pairs per step, warp-shuffle scans.
__global__ void __launch_bounds__(256) farRowKernel(FarRowLaunch L) {
    __shared__ double wsum[8];
    const uint32_t row = blockIdx.x, sample = L.firstSample + row;
    const float2 S = L.points[sample % L.Np];
    const int ls = int(sample / L.Np);
    const float gs = farSampleGain(L.gTab, L.cand, L.K, L.T, L.layers, sample % L.Np, ls);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t nE = L.C * L.slices;
    double* out = L.rowCdf + size_t(row) * nE;
    double carry = 0.0;
    for (uint32_t e0 = 0; e0 < nE; e0 += 256) {
        const uint32_t e = e0 + threadIdx.x;
        float w = 0.0f;
        if (e < nE) {
            const uint32_t c = e / L.slices, j = e - c * L.slices;
            const int kImg = imageLevel(ls, int(L.layers), j);
            const float4 cl = L.cell[c];
            const float* mass = L.cellMass + size_t(c) * L.layers;
            const float* gc = L.gCell + size_t(c) * L.layers;
            const float gmid = farMidGain(L, S, cl.x, cl.y);
            if (j == 0) L.gMid[size_t(row) * L.C + c] = gmid;
            for (uint32_t l = 0; l < L.layers; ++l) {
                const float mcl = mass[l];
                if (!(mcl > 0.0f)) continue;
                const float d2 = farDistance2(cl, S, int(l), kImg, L.h);
                w += farTerm(farSliceFactor(L.refl, j, int(l) - kImg, L.h, d2), mcl, d2, farMeanGain(gc[l], gs, gmid));
            }
        }
        double x = double(w);
        for (int o = 1; o < 32; o <<= 1) {
            const double y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        double base = carry, block = 0.0;
        for (int k = 0; k < 8; ++k) {
            if (k < warp) base += wsum[k];
            block += wsum[k];
        }
        if (e < nE) out[e] = base + x;
        carry += block;
        __syncthreads();
    }
}

// The K triangles nearest to every point (by centroid distance, ties by
// index): nearest first, and the same set by ascending index.
void buildCandidates(const std::vector<float2>& points, const std::vector<float2>& centroid, uint32_t K,
                     std::vector<uint32_t>& nearest, std::vector<uint32_t>& sorted, std::vector<uint32_t>& rank) {
    const uint32_t Np = uint32_t(points.size()), T = uint32_t(centroid.size());
    nearest.resize(size_t(Np) * K);
    sorted.resize(size_t(Np) * K);
    rank.resize(size_t(Np) * K);
    std::vector<std::pair<double, uint32_t>> d(T);
    std::vector<std::pair<uint32_t, uint32_t>> byTri(K);
    for (uint32_t pt = 0; pt < Np; ++pt) {
        for (uint32_t t = 0; t < T; ++t) {
            const double dx = double(centroid[t].x) - points[pt].x, dy = double(centroid[t].y) - points[pt].y;
            d[t] = {dx * dx + dy * dy, t};
        }
        std::partial_sort(d.begin(), d.begin() + K, d.end());
        for (uint32_t k = 0; k < K; ++k) {
            nearest[size_t(pt) * K + k] = d[k].second;
            byTri[k] = {d[k].second, k};
        }
        std::sort(byTri.begin(), byTri.end());
        for (uint32_t k = 0; k < K; ++k) {
            sorted[size_t(pt) * K + k] = byTri[k].first;
            rank[size_t(pt) * K + k] = byTri[k].second;
        }
    }
}

constexpr double kFarCellTriangles = 8.0;  // triangles per cell of the far prior's grid (bounding-box average)

// The far prior's cells: a square grid of side a over the triangle
// centroids' bounding box, a^2 = box area x kFarCellTriangles / T; the
// non-empty cells in row-major order, each with the mean centroid of its
// triangles and the softening (a/2)^2; the triangles of each cell ascending.
void buildFarCells(const std::vector<float2>& centroid, std::vector<uint32_t>& cellOf, std::vector<uint32_t>& cellStart,
                   std::vector<uint32_t>& cellTris, std::vector<float4>& cellXY) {
    const uint32_t T = uint32_t(centroid.size());
    double x0 = 1e300, x1 = -1e300, y0 = 1e300, y1 = -1e300;
    for (const float2& c : centroid) {
        x0 = std::min(x0, double(c.x));
        x1 = std::max(x1, double(c.x));
        y0 = std::min(y0, double(c.y));
        y1 = std::max(y1, double(c.y));
    }
    const double w = std::max(x1 - x0, 1e-12), hgt = std::max(y1 - y0, 1e-12);
    const double a = std::sqrt(w * hgt * kFarCellTriangles / double(std::max(T, 1u)));
    const uint32_t gx = uint32_t(std::min(4096.0, std::max(1.0, std::ceil(w / a))));
    const uint32_t gy = uint32_t(std::min(4096.0, std::max(1.0, std::ceil(hgt / a))));
    std::vector<uint32_t> grid(T);
    for (uint32_t t = 0; t < T; ++t) {
        const uint32_t ix = std::min(gx - 1, uint32_t(std::max(0.0, (double(centroid[t].x) - x0) / a)));
        const uint32_t iy = std::min(gy - 1, uint32_t(std::max(0.0, (double(centroid[t].y) - y0) / a)));
        grid[t] = iy * gx + ix;
    }
    std::vector<uint32_t> compact(size_t(gx) * gy, 0xffffffffu), count;
    std::vector<uint32_t> order(T);
    for (uint32_t t = 0; t < T; ++t) order[t] = t;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t u, uint32_t v) { return grid[u] < grid[v]; });
    cellOf.assign(T, 0);
    cellStart.clear();
    cellTris.assign(order.begin(), order.end());
    cellXY.clear();
    for (uint32_t i = 0; i < T; ++i) {
        const uint32_t t = order[i];
        if (compact[grid[t]] == 0xffffffffu) {
            compact[grid[t]] = uint32_t(cellStart.size());
            cellStart.push_back(i);
        }
        cellOf[t] = compact[grid[t]];
    }
    cellStart.push_back(T);
    const uint32_t C = uint32_t(cellStart.size() - 1);
    for (uint32_t c = 0; c < C; ++c) {
        double sx = 0.0, sy = 0.0;
        for (uint32_t i = cellStart[c]; i < cellStart[c + 1]; ++i) {
            sx += centroid[cellTris[i]].x;
            sy += centroid[cellTris[i]].y;
        }
        const double n = double(cellStart[c + 1] - cellStart[c]);
        cellXY.push_back(make_float4(float(sx / n), float(sy / n), float(0.25 * a * a), 0.0f));
    }
}

// The importance kernel's line order: for every sample level ls, the lines
// q = l * slices + j (layer l, reflection slice j) by increasing distance
// |l + 1/2 - kImg| to the image level (ties by q).  A line crosses about that
// many level planes along its 2-D path, so the lines of one lane slot of a
// team cross similar numbers of planes per triangle.
void buildLineOrder(uint32_t layers, uint32_t slices, std::vector<uint16_t>& ord) {
    const uint32_t n = slices * layers;
    ord.resize(size_t(layers + 1) * n);
    std::vector<std::pair<double, uint32_t>> key(n);
    for (uint32_t ls = 0; ls <= layers; ++ls) {
        for (uint32_t q = 0; q < n; ++q) {
            const uint32_t l = q / slices, j = q % slices;
            const int L = int(layers), s = int(ls);
            const int kImg = j == 1 ? -s : j == 2 ? 2 * L - s : j == 3 ? s - 2 * L : j == 4 ? s + 2 * L : s;
            key[q] = {std::fabs(double(l) + 0.5 - double(kImg)), q};
        }
        std::sort(key.begin(), key.end());
        for (uint32_t i = 0; i < n; ++i) ord[size_t(ls) * n + i] = uint16_t(key[i].second);
    }
}

}  // namespace

struct hase_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    uint32_t Np = 0, T = 0, L = 0, layers = 0, P = 0;
    double h = 0, nTot = 0, tau = 0, cladAbs = 0, extent = 0;
    uint32_t cladNumber = 0;
    std::vector<uint32_t> cladTypes;
    bool hasClad = false;  // some prism is cladding
    std::vector<double> betaCells, sigmaA, sigmaE;
    bool hasReflect = false;
    float tirCos2[2] = {-1.0f, -1.0f};
    DevBuf<float4> tri, walk, geo;
    DevBuf<int4> verts;
    DevBuf<uint16_t> lineOrder[2];  // importance line order per sample level: 1 and 5 reflection slices
    // local proposal (hase_context_set_local_proposal): per point the K
    // triangles nearest to it (by centroid distance, nearest first) and the
    // same set by ascending index; the far proposal's prefix of beta V over
    // the prisms and each point's candidate share of it, per beta version
    bool gridProposal = false;  // coarse-grid weights instead of the importance walks
    uint32_t localK = 0;
    float farFraction = 0.0f;
    DevBuf<uint32_t> candTri, candSorted, candRank;
    // the far prior: triangle cells (once per mesh), their beta V tables
    // (once per beta version), and the cell prefixes of a chunk's rows
    uint32_t farCells = 0;
    DevBuf<uint32_t> cellOf, cellStart, cellTris;
    DevBuf<float4> cellXY;
    DevBuf<float> cellMass, triPrefix, gCell, farMid, farColGrid;
    DevBuf<double> farRow;
    uint64_t farVersion = 0;
    DevBuf<float2> centroid, points, spec;
    DevBuf<float> gainBeta, srcBeta, reflect;
    DevBuf<float> gTab;  // g of every prism for the spectrally averaged (A, B) of the last solve
    // workspace
    DevBuf<float> lnw;
    DevBuf<uint32_t> q, offsets, activeA, activeB, counter, accTotal, accDrop, pDrop;
    DevBuf<unsigned int> itemCounter;
    uint32_t persistentBlocks = 0;  // resident rayKernel blocks on the device
    uint32_t variantBlocks[3][16] = {};  // the same for every walk mode x launch shape of kRayVariants (at most 16)
    DevBuf<unsigned long long> Q, accCross, pCross;
    DevBuf<double> accSum, accSum2, pSum, pSum2, mse;
    DevBuf<float> phi;
    // host copies used by the learned proposal's features
    std::vector<float2> hCentroid, hPoints;
    std::vector<float> hArea, hGainBeta, hReflect;
    std::vector<double> hBeta;  // betaVolume as given (FP64)
    // learned proposal: coarse gain grid, fallback rows, contribution log
    DevBuf<float> featGrid, logBuf, priorBuf;
    // the feature grid's layout (beta-independent, built on first use): grid
    // extents, the triangles (ascending) whose centre lies in each cell, and
    // the fill order of the empty cells, sweep by sweep
    bool featLayout = false;
    uint32_t featGx = 0, featGy = 0, featSweeps = 0;
    float featX0 = 0.0f, featY0 = 0.0f, featCellSize = 0.0f, featR = 0.0f;
    double featLnRb = 0.0, featLnRt = 0.0, featVmean = 0.0;
    DevBuf<uint32_t> featCellStart, featCellTris, featFill, featSweepStart;
    uint64_t betaVersion = 1;       // bumped by every beta upload
    uint64_t featVersion = 0;       // beta version the cached feature view was built for
    double featA = 0.0, featB = 0.0;
    ProposalView featView{};        // the cached feature view
    DevBuf<uint32_t> rowList;

    MeshView view() const {
        MeshView v{};
        invariantDivisor(T, v.divTm, v.divTs);
        invariantDivisor(Np, v.divNpm, v.divNps);
        v.tri = tri.p;
        v.walk = walk.p;
        v.geo = geo.p;
        v.verts = verts.p;
        v.centroid = centroid.p;
        v.gainBeta = gainBeta.p;
        v.gTab = gTab.p;
        v.srcBeta = srcBeta.p;
        v.points = points.p;
        v.reflect = hasReflect ? reflect.p : nullptr;
        v.lineOrder[0] = lineOrder[0].p;
        v.lineOrder[1] = lineOrder[1].p;
        v.T = T;
        v.layers = layers;
        v.P = P;
        v.Np = Np;
        v.h = float(h);
        v.cladAbs = float(cladAbs);
        v.tolEnd = float(4e-6 * extent);
        v.tirCos2[0] = tirCos2[0];
        v.tirCos2[1] = tirCos2[1];
        return v;
    }
};

namespace {

hase_status uploadBeta(hase_context* c, const double* betaVolume) {
    std::vector<float> gain(c->P), src(c->P);
    for (uint32_t p = 0; p < c->P; ++p) {
        const double b = betaVolume[p];
        if (!std::isfinite(b)) return fail(HASE_INVALID_ARGUMENT, "betaVolume[%u] is not finite", p);
        const uint32_t t = p % c->T;
        const bool clad = !c->cladTypes.empty() && c->cladTypes[t] == c->cladNumber;
        src[p] = float(b);
        gain[p] = clad ? NAN : float(b);
    }
    c->hGainBeta = gain;
    c->hBeta.assign(betaVolume, betaVolume + c->P);
    ++c->betaVersion;
    HASE_CUDA(cudaMemcpyAsync(c->gainBeta.p, gain.data(), c->P * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    HASE_CUDA(cudaMemcpyAsync(c->srcBeta.p, src.data(), c->P * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    HASE_CUDA(cudaStreamSynchronize(c->stream));
    return HASE_OK;
}

uint32_t adaptiveTarget(uint32_t minRays, uint32_t maxRays, uint32_t steps, uint32_t k) {
    // include/core/types.hpp:333-354: geometric growth minRays -> maxRays in `steps` increases.
    if (maxRays <= minRays || steps == 0) return minRays;
    if (k >= steps) return maxRays;
    const double growth = std::pow(double(maxRays) / double(minRays), 1.0 / double(steps));
    const double target = double(minRays) * std::pow(growth, double(k));
    const uint32_t r = uint32_t(std::ceil(target));
    return std::min(std::max(r, minRays), maxRays);
}

hase_status setDevice(hase_context* c) {
    HASE_CUDA(cudaSetDevice(c->device));
    return HASE_OK;
}

// Local proposal: candidate lists for the set K (once), and the far tables
// of the current beta (one prefix kernel and one per-point kernel on the
// context's stream, once per beta version).
hase_status prepareLocal(hase_context* c) {
    if (c->candTri.n != size_t(c->Np) * c->localK) {
        std::vector<uint32_t> nearest, sorted, rank;
        buildCandidates(c->hPoints, c->hCentroid, c->localK, nearest, sorted, rank);
        c->candTri.release();
        c->candSorted.release();
        c->candRank.release();
        HASE_CUDA(c->candTri.ensure(nearest.size()));
        HASE_CUDA(c->candSorted.ensure(sorted.size()));
        HASE_CUDA(c->candRank.ensure(rank.size()));
        HASE_CUDA(cudaMemcpy(c->candTri.p, nearest.data(), nearest.size() * 4, cudaMemcpyHostToDevice));
        HASE_CUDA(cudaMemcpy(c->candSorted.p, sorted.data(), sorted.size() * 4, cudaMemcpyHostToDevice));
        HASE_CUDA(cudaMemcpy(c->candRank.p, rank.data(), rank.size() * 4, cudaMemcpyHostToDevice));
    }
    if (c->localK >= c->T) return HASE_OK;  // every triangle is a candidate: no far rays
    if (c->farCells == 0) {
        std::vector<uint32_t> cellOf, cellStart, cellTris;
        std::vector<float4> cellXY;
        buildFarCells(c->hCentroid, cellOf, cellStart, cellTris, cellXY);
        const uint32_t C = uint32_t(cellXY.size());
        HASE_CUDA(c->cellOf.ensure(cellOf.size()));
        HASE_CUDA(c->cellStart.ensure(cellStart.size()));
        HASE_CUDA(c->cellTris.ensure(cellTris.size()));
        HASE_CUDA(c->cellXY.ensure(C));
        HASE_CUDA(c->cellMass.ensure(size_t(C) * c->layers));
        HASE_CUDA(c->gCell.ensure(size_t(C) * c->layers));
        HASE_CUDA(c->triPrefix.ensure(c->P));
        HASE_CUDA(cudaMemcpy(c->cellOf.p, cellOf.data(), cellOf.size() * 4, cudaMemcpyHostToDevice));
        HASE_CUDA(cudaMemcpy(c->cellStart.p, cellStart.data(), cellStart.size() * 4, cudaMemcpyHostToDevice));
        HASE_CUDA(cudaMemcpy(c->cellTris.p, cellTris.data(), cellTris.size() * 4, cudaMemcpyHostToDevice));
        HASE_CUDA(cudaMemcpy(c->cellXY.p, cellXY.data(), C * sizeof(float4), cudaMemcpyHostToDevice));
        c->farCells = C;
        c->farVersion = 0;
    }
    if (c->farVersion != c->betaVersion) {
        const uint32_t n = c->farCells * c->layers;
        farCellKernel<<<(n + 255) / 256, 256, 0, c->stream>>>(c->cellStart.p, c->cellTris.p, c->farCells, c->srcBeta.p,
                                                              c->geo.p, c->T, c->layers, float(c->h), c->cellMass.p,
                                                              c->triPrefix.p);
        HASE_CUDA(cudaGetLastError());
        c->farVersion = c->betaVersion;
    }
    return HASE_OK;
}

// The far prior's surface factors: each surface's mean reflectivity (at
// least 1/4) and its total-internal-reflection bound on uz^2.
void farSlicePrior(const hase_context* c, FarSlices& f) {
    double R[2] = {0.0, 0.0};
    if (c->hasReflect && !c->hReflect.empty())
        for (uint32_t t = 0; t < c->T; ++t)
            for (int s = 0; s < 2; ++s) R[s] += double(c->hReflect[2 * t + s]) / double(c->T);
    for (int s = 0; s < 2; ++s) {
        f.R[s] = float(std::max(R[s], 0.25));
        f.tir[s] = c->tirCos2[s];
    }
}

// The far prior's view of a context for a solve of `slices` reflection
// slices (rowCdf: the chunk's row prefixes).
FarView farView(const hase_context* c, uint32_t slices) {
    FarView f{};
    f.slices = slices;
    farSlicePrior(c, f.refl);
    f.cellOf = c->cellOf.p;
    f.cellStart = c->cellStart.p;
    f.cellTris = c->cellTris.p;
    f.cell = c->cellXY.p;
    f.cellMass = c->cellMass.p;
    f.triPrefix = c->triPrefix.p;
    f.gCell = c->gCell.p;
    f.rowCdf = c->farRow.p;
    f.gMid = c->farMid.p;
    f.C = c->farCells;
    return f;
}

// Entries of a sample's weight row: every (slice, prism), or with the local
// proposal the (slice, layer, candidate) entries.
uint32_t rowEntries(const hase_context* c, uint32_t slices) {
    return c->localK ? slices * c->layers * c->localK : slices * c->P;
}

// The local proposal's candidate fields of a launch's views.
void localFields(hase_context* c, ProposalView& pv) {
    if (!c->localK) return;
    pv.cand = c->candTri.p;
    pv.K = c->localK;
    invariantDivisor(c->localK, pv.divKm, pv.divKs);
}
void localFields(hase_context* c, ImportanceLaunch& il) {
    if (!c->localK) return;
    il.cand = c->candTri.p;
    il.K = c->localK;
}

struct LearnedArgs {
    hase_proposal* net;
    float alpha;             // weight of the beta V / d^2 prior in the mixture
    float fallbackVariance;  // per-ray relative variance that sends a sample to the exact weights (0: never)
    uint32_t fallbackSamples;
};

constexpr uint32_t kGridCells = 48;  // feature grid cells along the longer side

// Mean gain coefficient g = A beta - B (-claddingAbsorption in cladding) of
// the prisms of one layer (block) whose centre falls in each grid cell, then
// the empty cells filled from their filled 4-neighbours, sweep by sweep (a
// cell filled in a sweep is read from the next sweep on).  The sums run in
// ascending triangle order and in the neighbour order of the layout.
__global__ void featureGridKernel(const float* gainBeta, uint32_t T, double A, double B, float cladAbs,
                                  const uint32_t* cellStart, const uint32_t* cellTris, uint32_t cells,
                                  const uint32_t* fill, const uint32_t* sweepStart, uint32_t sweeps, float* grid) {
    const uint32_t l = blockIdx.x;
    float* gl = grid + size_t(l) * cells;
    const float* bl = gainBeta + size_t(l) * T;
    for (uint32_t k = threadIdx.x; k < cells; k += blockDim.x) {
        const uint32_t a = cellStart[k], e = cellStart[k + 1];
        if (a == e) continue;  // empty: filled below
        float sum = 0.0f;
        for (uint32_t i = a; i < e; ++i) {
            const float bt = bl[cellTris[i]];
            sum += bt != bt ? -cladAbs : float(A * double(bt) - B);
        }
        gl[k] = sum / float(e - a);
    }
    __syncthreads();
    for (uint32_t sw = 0; sw < sweeps; ++sw) {
        for (uint32_t e = sweepStart[sw] + threadIdx.x; e < sweepStart[sw + 1]; e += blockDim.x) {
            const uint32_t* f = fill + 6 * size_t(e);  // cell, neighbours n, up to 4 neighbour cells
            float add = 0.0f;
            for (uint32_t i = 0; i < f[1]; ++i) add += gl[f[2 + i]];
            gl[f[0]] = add / float(f[1]);
        }
        __syncthreads();
    }
}

// The feature grid's layout, once per mesh (host; it does not depend on beta).
hase_status buildFeatureLayout(hase_context* c) {
    float x0 = INFINITY, y0 = INFINITY, x1 = -INFINITY, y1 = -INFINITY, R = 0.0f;
    for (const float2& q : c->hPoints) {
        x0 = std::min(x0, q.x);
        y0 = std::min(y0, q.y);
        x1 = std::max(x1, q.x);
        y1 = std::max(y1, q.y);
        R = std::max(R, std::sqrt(q.x * q.x + q.y * q.y));
    }
    const float cell = std::max(x1 - x0, y1 - y0) / float(kGridCells) * 1.0001f;
    const uint32_t gx = uint32_t(std::ceil((x1 - x0) / cell)) + 1, gy = uint32_t(std::ceil((y1 - y0) / cell)) + 1;
    const uint32_t cells = gx * gy;
    std::vector<uint32_t> cellOf(c->T), start(cells + 1, 0), tris(c->T);
    for (uint32_t t = 0; t < c->T; ++t) {
        const uint32_t ix = std::min(gx - 1, uint32_t((c->hCentroid[t].x - x0) / cell));
        const uint32_t iy = std::min(gy - 1, uint32_t((c->hCentroid[t].y - y0) / cell));
        cellOf[t] = iy * gx + ix;
        ++start[cellOf[t] + 1];
    }
    for (uint32_t k = 0; k < cells; ++k) start[k + 1] += start[k];
    std::vector<uint32_t> pos(start.begin(), start.end() - 1);
    for (uint32_t t = 0; t < c->T; ++t) tris[pos[cellOf[t]]++] = t;  // ascending t within each cell
    // fill order: every sweep fills the empty cells with a filled 4-neighbour
    // (+x, -x, +y, -y), from the cells filled before the sweep
    std::vector<uint8_t> filled(cells);
    for (uint32_t k = 0; k < cells; ++k) filled[k] = start[k + 1] > start[k];
    std::vector<uint32_t> fill, sweepStart{0};
    for (uint32_t sweep = 0; sweep < gx + gy; ++sweep) {
        std::vector<uint32_t> now;
        for (uint32_t iy = 0; iy < gy; ++iy)
            for (uint32_t ix = 0; ix < gx; ++ix) {
                const uint32_t k = iy * gx + ix;
                if (filled[k]) continue;
                uint32_t e[6] = {k, 0, 0, 0, 0, 0};
                const int dxy[4][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}};
                for (auto& o : dxy) {
                    const int jx = int(ix) + o[0], jy = int(iy) + o[1];
                    if (jx < 0 || jy < 0 || jx >= int(gx) || jy >= int(gy)) continue;
                    const uint32_t kk = uint32_t(jy) * gx + uint32_t(jx);
                    if (filled[kk]) e[2 + e[1]++] = kk;
                }
                if (e[1] == 0) continue;
                fill.insert(fill.end(), e, e + 6);
                now.push_back(k);
            }
        if (now.empty()) break;
        for (uint32_t k : now) filled[k] = 1;
        sweepStart.push_back(uint32_t(fill.size() / 6));
    }
    HASE_CUDA(c->featCellStart.ensure(cells + 1));
    HASE_CUDA(c->featCellTris.ensure(std::max<uint32_t>(c->T, 1)));
    HASE_CUDA(c->featFill.ensure(std::max<size_t>(fill.size(), 6)));
    HASE_CUDA(c->featSweepStart.ensure(sweepStart.size()));
    HASE_CUDA(cudaMemcpy(c->featCellStart.p, start.data(), start.size() * 4, cudaMemcpyHostToDevice));
    HASE_CUDA(cudaMemcpy(c->featCellTris.p, tris.data(), tris.size() * 4, cudaMemcpyHostToDevice));
    if (!fill.empty()) HASE_CUDA(cudaMemcpy(c->featFill.p, fill.data(), fill.size() * 4, cudaMemcpyHostToDevice));
    HASE_CUDA(cudaMemcpy(c->featSweepStart.p, sweepStart.data(), sweepStart.size() * 4, cudaMemcpyHostToDevice));
    double lnRb = 0.0, lnRt = 0.0, vmean = 0.0;
    if (!c->hReflect.empty()) {
        for (uint32_t t = 0; t < c->T; ++t) {
            lnRb += std::log(std::max(1e-6, double(c->hReflect[2 * t]))) / c->T;
            lnRt += std::log(std::max(1e-6, double(c->hReflect[2 * t + 1]))) / c->T;
        }
    }
    for (float a : c->hArea) vmean += double(a) * c->h / c->T;
    c->featGx = gx;
    c->featGy = gy;
    c->featSweeps = uint32_t(sweepStart.size() - 1);
    c->featX0 = x0;
    c->featY0 = y0;
    c->featCellSize = cell;
    c->featR = R;
    c->featLnRb = lnRb;
    c->featLnRt = lnRt;
    c->featVmean = vmean;
    c->featLayout = true;
    return HASE_OK;
}

// Feature view of the context: the coarse gain grid (mean g = A beta - B of
// the prisms whose centre falls in a cell, empty cells filled from their
// neighbours; built on the device from the resident beta), scales, and mean
// reflectivities.
hase_status buildProposalView(hase_context* c, double A, double B, ProposalView& V) {
    if (!c->featLayout) HASE_TRY(buildFeatureLayout(c));
    const uint32_t cells = c->featGx * c->featGy, L = c->layers;
    HASE_CUDA(c->featGrid.ensure(size_t(L) * cells));
    featureGridKernel<<<L, 256, 0, c->stream>>>(c->gainBeta.p, c->T, A, B, float(c->cladAbs), c->featCellStart.p,
                                                 c->featCellTris.p, cells, c->featFill.p, c->featSweepStart.p,
                                                 c->featSweeps, c->featGrid.p);
    HASE_CUDA(cudaGetLastError());
    V = ProposalView{};
    V.m = c->view();
    V.grid = c->featGrid.p;
    V.gx = c->featGx;
    V.gy = c->featGy;
    V.x0 = c->featX0;
    V.y0 = c->featY0;
    V.invCell = 1.0f / c->featCellSize;
    V.lnRb = float(c->featLnRb);
    V.lnRt = float(c->featLnRt);
    V.R = std::max(c->featR, 1e-6f);
    V.H = float(c->h * L);
    V.invR = 1.0f / V.R;
    V.invH = 1.0f / V.H;
    V.invTwoH = 0.5f / V.H;
    V.invh = float(1.0 / c->h);
    V.lnVref = float(std::log(std::max(c->featVmean, 1e-30) / (double(V.R) * V.R)));
    const double se = (A - B), sa = B;
    V.lnSigmaRatio = float(std::log(std::max(se, 1e-30) / std::max(sa, 1e-30)));
    return HASE_OK;
}

// The feature view, rebuilt (one kernel on the context's stream) only when
// beta or the averaged spectrum changed.
hase_status cachedProposalView(hase_context* c, double A, double B, ProposalView& V) {
    if (c->featVersion == c->betaVersion && c->featA == A && c->featB == B) {
        V = c->featView;
        return HASE_OK;
    }
    HASE_TRY(buildProposalView(c, A, B, V));
    c->featView = V;
    c->featVersion = c->betaVersion;
    c->featA = A;
    c->featB = B;
    return HASE_OK;
}

}  // namespace

extern "C" {

const char* hase_last_error_message(void) { return g_lastError.c_str(); }

int hase_abi_version(void) { return HASE_B200_ABI_VERSION; }

const char* hase_status_string(hase_status s) {
    switch (s) {
        case HASE_OK: return "ok";
        case HASE_INVALID_ARGUMENT: return "invalid argument";
        case HASE_CUDA_ERROR: return "CUDA error";
        case HASE_OUT_OF_MEMORY: return "out of device memory";
        case HASE_DEVICE_TIMEOUT: return "device timeout";
        case HASE_DROPPED_RAYS: return "dropped rays";
        case HASE_NOT_CONVERGED: return "not converged";
        case HASE_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

int hase_ray_kernel_variant_count(void) { return int(kNumRayVariants); }

const char* hase_ray_kernel_variant_name(uint32_t variant) {
    return variant < kNumRayVariants ? kRayVariants[variant].name : "";
}

hase_status hase_context_create(const hase_mesh_desc* d, const hase_spectrum_desc* sp, int device,
                                hase_context** out) {
    if (!d || !sp || !out) return fail(HASE_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (d->numberOfLevels < 2) return fail(HASE_INVALID_ARGUMENT, "numberOfLevels must be >= 2");
    if (d->numberOfTriangles == 0 || d->numberOfPoints < 3) return fail(HASE_INVALID_ARGUMENT, "empty mesh");
    if (!d->points || !d->triangles || !d->betaVolume) return fail(HASE_INVALID_ARGUMENT, "mesh arrays missing");
    if (!(d->thickness > 0.0)) return fail(HASE_INVALID_ARGUMENT, "thickness must be positive");
    if (!(d->nTot > 0.0) || !(d->crystalTFluo > 0.0)) return fail(HASE_INVALID_ARGUMENT, "nTot and crystalTFluo must be positive");
    if (sp->numberOfWavelengths == 0 || !sp->sigmaA || !sp->sigmaE) return fail(HASE_INVALID_ARGUMENT, "empty spectrum");
    if (uint64_t(d->numberOfTriangles) * (d->numberOfLevels - 1) * 5ull >= (1ull << 31))
        return fail(HASE_INVALID_ARGUMENT, "mesh too large");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(HASE_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= count) return fail(HASE_INVALID_ARGUMENT, "device %d out of range", device);

    hase_context* c = new (std::nothrow) hase_context();
    if (!c) return fail(HASE_OUT_OF_MEMORY, "host allocation failed");
    auto cleanup = [&](hase_status s) {
        hase_context_destroy(c);
        return s;
    };
    c->device = device;
    c->Np = d->numberOfPoints;
    c->T = d->numberOfTriangles;
    c->L = d->numberOfLevels;
    c->layers = c->L - 1;
    c->P = c->T * c->layers;
    c->h = d->thickness;
    c->nTot = d->nTot;
    c->tau = d->crystalTFluo;
    c->cladAbs = d->claddingAbsorption;
    c->cladNumber = d->claddingNumber;
    if (d->claddingCellTypes) c->cladTypes.assign(d->claddingCellTypes, d->claddingCellTypes + c->T);
    c->hasClad = std::find(c->cladTypes.begin(), c->cladTypes.end(), c->cladNumber) != c->cladTypes.end();
    if (d->betaCells) c->betaCells.assign(d->betaCells, d->betaCells + size_t(c->Np) * c->L);
    c->sigmaA.assign(sp->sigmaA, sp->sigmaA + sp->numberOfWavelengths);
    c->sigmaE.assign(sp->sigmaE, sp->sigmaE + sp->numberOfWavelengths);
    for (uint32_t l = 0; l < sp->numberOfWavelengths; ++l)
        if (!std::isfinite(sp->sigmaA[l]) || !std::isfinite(sp->sigmaE[l]) || sp->sigmaA[l] < 0 || sp->sigmaE[l] < 0)
            return cleanup(fail(HASE_INVALID_ARGUMENT, "cross sections must be finite and non-negative"));
    if (d->refractiveIndices) {
        for (int s = 0; s < 2; ++s) {
            const double nin = d->refractiveIndices[2 * s], nout = d->refractiveIndices[2 * s + 1];
            if (nout < nin && nin > 0) {
                const double r = nout / nin;
                c->tirCos2[s] = float(1.0 - r * r);
            }
        }
    }
    HostTables ht;
    hase_status st = buildHostTables(d, ht, c->extent);
    if (st != HASE_OK) return cleanup(st);
    c->extent = std::max(c->extent, c->h * c->layers);
    c->hCentroid = ht.centroid;
    c->hPoints = ht.points;
    c->hArea.resize(c->T);
    for (uint32_t t = 0; t < c->T; ++t) c->hArea[t] = ht.geo[2 * t + 1].z;
    if (d->reflectivities)
        for (size_t k = 0; k < 2 * size_t(c->T); ++k) c->hReflect.push_back(float(d->reflectivities[k]));

    if (cudaSetDevice(device) != cudaSuccess) return cleanup(fail(HASE_CUDA_ERROR, "cudaSetDevice failed"));
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        return cleanup(fail(HASE_CUDA_ERROR, "cudaStreamCreate failed"));
    for (auto& e : c->ev)
        if (cudaEventCreate(&e) != cudaSuccess) return cleanup(fail(HASE_CUDA_ERROR, "cudaEventCreate failed"));
    auto up = [&](auto& buf, const auto& vec) -> hase_status {
        using T = typename std::decay_t<decltype(vec)>::value_type;
        HASE_CUDA(buf.ensure(vec.size()));
        HASE_CUDA(cudaMemcpyAsync(buf.p, vec.data(), vec.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
        return HASE_OK;
    };
    if ((st = up(c->tri, ht.tri)) != HASE_OK) return cleanup(st);
    if ((st = up(c->walk, ht.walk)) != HASE_OK) return cleanup(st);
    if ((st = up(c->geo, ht.geo)) != HASE_OK) return cleanup(st);
    if ((st = up(c->verts, ht.verts)) != HASE_OK) return cleanup(st);
    if (uint64_t(5) * c->layers < 65536) {  // importance line order (16-bit line indices)
        for (int r = 0; r < 2; ++r) {
            std::vector<uint16_t> ord;
            buildLineOrder(c->layers, r ? 5u : 1u, ord);
            if ((st = up(c->lineOrder[r], ord)) != HASE_OK) return cleanup(st);
        }
    }
    if ((st = up(c->centroid, ht.centroid)) != HASE_OK) return cleanup(st);
    if ((st = up(c->points, ht.points)) != HASE_OK) return cleanup(st);
    if (c->gainBeta.ensure(c->P) != cudaSuccess || c->srcBeta.ensure(c->P) != cudaSuccess)
        return cleanup(fail(HASE_OUT_OF_MEMORY, "beta tables"));
    if (d->reflectivities) {
        std::vector<float> r(2 * size_t(c->T));
        for (size_t i = 0; i < r.size(); ++i) r[i] = float(d->reflectivities[i]);
        c->hasReflect = true;
        if ((st = up(c->reflect, r)) != HASE_OK) return cleanup(st);
    }
    if ((st = uploadBeta(c, d->betaVolume)) != HASE_OK) return cleanup(st);
    {  // resident spectrum and launch shape: hase_estimate_sample_noalloc allocates nothing
        std::vector<float2> spec(c->sigmaA.size());
        for (size_t l = 0; l < spec.size(); ++l)
            spec[l] = make_float2(float(c->nTot * (c->sigmaE[l] + c->sigmaA[l])), float(c->nTot * c->sigmaA[l]));
        if ((st = up(c->spec, spec)) != HASE_OK) return cleanup(st);
    }
    {
        int perSM = 0, sms = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, rayKernel<kRayBlock, kRefill, kRayMinBlocks>,
                                                          kRayBlock, 0) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
            return cleanup(fail(HASE_CUDA_ERROR, "occupancy query failed"));
        c->persistentBlocks = uint32_t(std::max(1, perSM) * std::max(1, sms));
    }
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return cleanup(fail(HASE_CUDA_ERROR, "upload failed"));
    *out = c;
    return HASE_OK;
}

hase_status hase_context_update_beta(hase_context* c, const double* betaVolume, const double* betaCells) {
    if (!c || !betaVolume) return fail(HASE_INVALID_ARGUMENT, "null argument");
    HASE_TRY(setDevice(c));
    HASE_TRY(uploadBeta(c, betaVolume));
    if (betaCells) c->betaCells.assign(betaCells, betaCells + size_t(c->Np) * c->L);
    return HASE_OK;
}

// Default share of the far prior's rays: measured best of 0.25 / 0.5 / 0.75 /
// 0.9 for K = 16, 64 and 256 on a 18,816-triangle x 29-layer disc with 8
// wavelengths and reflections (relative variance per ray 0.21 against 0.14 of
// the full proposal).
constexpr float kDefaultFarFraction = 0.9f;

hase_status hase_context_set_grid_proposal(hase_context* c, uint32_t enable) {
    if (!c) return fail(HASE_INVALID_ARGUMENT, "null context");
    c->gridProposal = enable != 0;
    return HASE_OK;
}

hase_status hase_context_set_local_proposal(hase_context* c, uint32_t triangles, float farFraction) {
    if (!c) return fail(HASE_INVALID_ARGUMENT, "null context");
    if (!(farFraction >= 0.0f) || farFraction >= 1.0f) return fail(HASE_INVALID_ARGUMENT, "farFraction must be in [0, 1)");
    if (uint64_t(triangles) * c->layers * 5u >= (1ull << 31))
        return fail(HASE_INVALID_ARGUMENT, "too many local triangles for this mesh");
    c->localK = std::min(triangles, c->T);
    c->farFraction = farFraction > 0.0f ? farFraction : kDefaultFarFraction;
    return HASE_OK;
}

hase_status hase_context_destroy(hase_context* c) {
    if (!c) return HASE_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return HASE_OK;
}

// The adaptive solve of hase_calc_phi_ase.  la != null: the learned
// proposal replaces the importance weights (samples whose first-pass per-ray
// relative variance exceeds la->fallbackVariance restart with the importance
// weights).  logOut != null: the rays' contributions are summed per
// (sample, slice, prism) into logOut [samples][slices * P].
static hase_status calcCore(hase_context* c, const hase_experiment_desc* ex, const hase_compute_desc* cp,
                            hase_result* res, LearnedArgs* la, float* logOut) {
    if (!c || !ex || !cp || !res) return fail(HASE_INVALID_ARGUMENT, "null argument");
    HASE_TRY(setDevice(c));
    const uint32_t nSamplesTotal = c->Np * c->L;
    const uint32_t first = cp->minSample;
    const uint32_t last = cp->maxSample == UINT32_MAX ? nSamplesTotal - 1 : cp->maxSample;
    if (first > last || last >= nSamplesTotal)
        return fail(HASE_INVALID_ARGUMENT, "sample range [%u, %u] outside [0, %u)", first, last, nSamplesTotal);
    if (ex->minRays == 0) return fail(HASE_INVALID_ARGUMENT, "minRays must be positive");
    if (ex->maxRays != 0 && ex->maxRays < ex->minRays) return fail(HASE_INVALID_ARGUMENT, "maxRays < minRays");
    if (!(ex->mseThreshold >= 0.0)) return fail(HASE_INVALID_ARGUMENT, "mseThreshold must be >= 0");
    const uint32_t maxRays = std::max(ex->maxRays, ex->minRays);
    const uint32_t nS = last - first + 1;
    const uint32_t slices = ex->useReflections ? 5u : 1u;
    // local proposal: a row holds the point's K candidate triangles x layers
    // x slices; the rest of the medium is sampled by the far rays
    const bool local = c->localK > 0;
    const uint32_t K = c->localK;
    const uint32_t nW = local ? slices * c->layers * K : slices * c->P;
    if (local) HASE_TRY(prepareLocal(c));
    uint32_t divKm = 0, divKs = 0;
    if (local) invariantDivisor(K, divKm, divKs);

    // spectrum: (A, B) per wavelength, g = beta*A - B
    const uint32_t nLambda = ex->monochromatic ? 1u : uint32_t(c->sigmaA.size());
    std::vector<float2> spec(nLambda);
    double meanA = 0, meanB = 0, maxSA = 0, maxSE = 0;
    for (uint32_t l = 0; l < nLambda; ++l) {
        const double A = c->nTot * (c->sigmaE[l] + c->sigmaA[l]), B = c->nTot * c->sigmaA[l];
        spec[l] = make_float2(float(A), float(B));
        meanA += A / nLambda;
        meanB += B / nLambda;
        maxSA = std::max(maxSA, c->sigmaA[l]);
        maxSE = std::max(maxSE, c->sigmaE[l]);
    }
    HASE_CUDA(c->spec.ensure(nLambda));
    HASE_CUDA(cudaMemcpyAsync(c->spec.p, spec.data(), nLambda * sizeof(float2), cudaMemcpyHostToDevice, c->stream));
    ProposalView pv{};
    uint32_t proposalGrid = 0;
    const bool gridWeights = c->gridProposal && !la;
    if (gridWeights) HASE_TRY(cachedProposalView(c, meanA, meanB, pv));
    if (la) {
        if (la->net->device != c->device)
            return fail(HASE_INVALID_ARGUMENT, "the proposal network and the context are on different devices");
        HASE_TRY(cachedProposalView(c, meanA, meanB, pv));
        HASE_CUDA(cudaFuncSetAttribute(proposalKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemBytes)));
        int sms = 0;
        HASE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
        proposalGrid = uint32_t(std::max(1, sms) * kMlpBlocksPerSM);
        la->fallbackSamples = 0;
    }

    // batch rows by the workspace budget
    const uint64_t budget = cp->workspaceBytes ? cp->workspaceBytes : (uint64_t(4) << 30);
    const bool farPrior = local && K < c->T;
    const uint64_t perRow = uint64_t(nW) * 12 + 16 + kMaxItems * 28ull + 64 + (farPrior ? uint64_t(c->farCells) * (slices * 8ull + 4ull) : 0ull);
    uint32_t rows = uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(nS, budget / perRow)));
    HASE_CUDA(c->lnw.ensure(size_t(rows) * nW));
    HASE_CUDA(c->q.ensure(size_t(rows) * nW));
    HASE_CUDA(c->offsets.ensure(size_t(rows) * (nW + 1)));
    HASE_CUDA(c->Q.ensure(rows));
    if (farPrior) {
        HASE_CUDA(c->farRow.ensure(size_t(rows) * c->farCells * slices));
        HASE_CUDA(c->farMid.ensure(size_t(rows) * c->farCells));
    }
    HASE_CUDA(c->activeA.ensure(rows));
    HASE_CUDA(c->activeB.ensure(rows));
    HASE_CUDA(c->counter.ensure(1));
    HASE_CUDA(c->itemCounter.ensure(1));
    if (!validImportanceLayers(cp->importanceLayers))
        return fail(HASE_INVALID_ARGUMENT, "importanceLayers must be 0, 2, 4 or 8");
    if (cp->rayKernelVariant >= kNumRayVariants)
        return fail(HASE_INVALID_ARGUMENT, "rayKernelVariant %u >= %u", cp->rayKernelVariant, kNumRayVariants);
    const uint32_t variant = cp->rayKernelVariant;
    if (c->variantBlocks[0][variant] == 0) {
        const RayVariant& v = kRayVariants[variant];
        int sms = 0;
        HASE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
        void (*const modes[3])(RayLaunch) = {v.kernel, v.mono, v.noClad};
        for (int w = 0; w < 3; ++w) {
            int perSM = 0;
            HASE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, modes[w], v.block, 0));
            c->variantBlocks[w][variant] = uint32_t(std::max(1, perSM) * std::max(1, sms));
        }
    }
    if (c->persistentBlocks == 0) {
        int perSM = 0, sms = 0;
        HASE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, rayKernel<kRayBlock, kRefill, kRayMinBlocks>, kRayBlock, 0));
        HASE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
        c->persistentBlocks = uint32_t(std::max(1, perSM) * std::max(1, sms));
    }
    HASE_CUDA(c->accSum.ensure(rows));
    HASE_CUDA(c->accSum2.ensure(rows));
    HASE_CUDA(c->accTotal.ensure(rows));
    HASE_CUDA(c->accDrop.ensure(rows));
    HASE_CUDA(c->accCross.ensure(rows));
    HASE_CUDA(c->phi.ensure(rows));
    HASE_CUDA(c->mse.ensure(rows));
    HASE_CUDA(c->pSum.ensure(size_t(rows) * kMaxItems));
    HASE_CUDA(c->pSum2.ensure(size_t(rows) * kMaxItems));
    HASE_CUDA(c->pDrop.ensure(size_t(rows) * kMaxItems));
    HASE_CUDA(c->pCross.ensure(size_t(rows) * kMaxItems));
    if (logOut) HASE_CUDA(c->logBuf.ensure(size_t(rows) * nW));
    if (la) {
        HASE_CUDA(c->rowList.ensure(rows));
        HASE_CUDA(c->priorBuf.ensure(size_t(rows) * nW));
    }
    std::vector<uint32_t> hList;
    std::vector<double> hRse;
    std::vector<uint32_t> hTot;

    // the importance walks, and the ray walk of a monochromatic solve, read
    // each prism's g from a table (rebuilt here: beta may have changed since
    // the last solve)
    // walk mode of the ray launches (the logging launches keep the general walk)
    const int walk = logOut ? kWalkBeta : (nLambda == 1 ? kWalkTable : (c->hasClad ? kWalkBeta : kWalkBetaNoClad));
    HASE_CUDA(c->gTab.ensure(c->P));
    gainTableKernel<<<(c->P + 255) / 256, 256, 0, c->stream>>>(c->gainBeta.p, float(meanA), float(meanB),
                                                               float(c->cladAbs), c->P, c->gTab.p);
    HASE_CUDA(cudaGetLastError());
    ProposalView fpv{};
    if (farPrior) {  // the far prior's cell gains for this solve's g, and the layer-averaged coarse gain grid
        const uint32_t n = c->farCells * c->layers;
        farGainKernel<<<(n + 255) / 256, 256, 0, c->stream>>>(c->cellStart.p, c->cellTris.p, c->farCells, c->gTab.p, c->T,
                                                              c->layers, c->gCell.p);
        HASE_CUDA(cudaGetLastError());
        HASE_TRY(cachedProposalView(c, meanA, meanB, fpv));
        const uint32_t cells = fpv.gx * fpv.gy;
        HASE_CUDA(c->farColGrid.ensure(cells));
        farColumnKernel<<<(cells + 255) / 256, 256, 0, c->stream>>>(fpv.grid, cells, c->layers, c->farColGrid.p);
        HASE_CUDA(cudaGetLastError());
    }
    const MeshView mv = c->view();
    const double C = c->nTot / (4.0 * kPi * c->tau);
    std::vector<float> hPhi(rows);
    std::vector<double> hMse(rows);
    std::vector<uint32_t> hTotal(rows), hDrop(rows);
    std::vector<unsigned long long> hCross(rows);
    res->raysTraced = 0;
    res->crossings = 0;
    res->importanceMilliseconds = 0;
    res->rayMilliseconds = 0;
    res->totalMilliseconds = 0;
    res->passes = 0;
    res->unconvergedSamples = 0;
    res->kernelLaunches = farPrior ? 3 : 1;  // the gain table (and the far prior's cell gains and gain grid)
    uint64_t droppedTotal = 0;

    for (uint32_t b0 = 0; b0 < nS; b0 += rows) {
        const uint32_t nRows = std::min(rows, nS - b0);
        const uint32_t firstSample = first + b0;
        HASE_CUDA(cudaEventRecord(c->ev[0], c->stream));
        ImportanceLaunch il{mv, firstSample, slices, nW, float(meanA), float(meanB), c->lnw.p, nullptr};
        il.cand = local ? c->candTri.p : nullptr;
        il.K = K;
        auto launchImportanceRows = [&](uint32_t nLaunchRows) {
            launchImportance(cp->importanceLayers, il, c->layers, c->T, nLaunchRows, c->stream, true);
        };
        if (la) {
            pv.firstSample = firstSample;
            pv.nW = nW;
            localFields(c, pv);
            ProposalLaunch pl{pv, la->net->wimg.p, la->net->vec.p, c->lnw.p, c->priorBuf.p, nullptr, nRows,
                              la->net->error.p};
            const uint64_t tiles = (uint64_t(nRows) * nW + kTile - 1) / kTile;
            proposalKernel<<<uint32_t(std::min<uint64_t>(tiles, proposalGrid)), kTile, kSmemBytes, c->stream>>>(pl);
            HASE_CUDA(cudaGetLastError());
            mixtureKernel<<<nRows, 1024, 0, c->stream>>>(nW, c->lnw.p, c->priorBuf.p, la->alpha);
            res->kernelLaunches += 1;
        } else if (gridWeights) {
            pv.firstSample = firstSample;
            pv.nW = nW;
            localFields(c, pv);
            const ProposalLaunch gl{pv, nullptr, nullptr, c->lnw.p, nullptr, nullptr, nRows, nullptr};
            HASE_CUDA(launchGridWeights(gl, c->stream));
        } else {
            launchImportanceRows(nRows);
        }
        if (farPrior) {  // the far prior's cell prefixes of the chunk's rows
            FarRowLaunch fl{c->cellXY.p, c->cellMass.p, c->gCell.p, c->gTab.p, c->candTri.p, c->farCells, slices,
                            c->layers, c->Np, firstSample, K, c->T, c->points.p, float(c->h), {}, c->farRow.p};
            fl.gMid = c->farMid.p;
            fl.colGrid = c->farColGrid.p;
            fl.gx = fpv.gx;
            fl.gy = fpv.gy;
            fl.x0 = fpv.x0;
            fl.y0 = fpv.y0;
            fl.invCell = fpv.invCell;
            farSlicePrior(c, fl.refl);
            farRowKernel<<<nRows, 256, 0, c->stream>>>(fl);
            res->kernelLaunches += 1;
        }
        HASE_CUDA(cudaGetLastError());
        if (logOut) HASE_CUDA(cudaMemsetAsync(c->logBuf.p, 0, size_t(nRows) * nW * sizeof(float), c->stream));
        HASE_CUDA(cudaEventRecord(c->ev[1], c->stream));
        HASE_CUDA(cudaMemsetAsync(c->accSum.p, 0, nRows * sizeof(double), c->stream));
        HASE_CUDA(cudaMemsetAsync(c->accSum2.p, 0, nRows * sizeof(double), c->stream));
        HASE_CUDA(cudaMemsetAsync(c->accTotal.p, 0, nRows * sizeof(uint32_t), c->stream));
        HASE_CUDA(cudaMemsetAsync(c->accDrop.p, 0, nRows * sizeof(uint32_t), c->stream));
        HASE_CUDA(cudaMemsetAsync(c->accCross.p, 0, nRows * sizeof(unsigned long long), c->stream));
        iotaKernel<<<(nRows + 255) / 256, 256, 0, c->stream>>>(c->activeA.p, nRows);
        HASE_CUDA(cudaGetLastError());
        res->kernelLaunches += 2;  // importance + iota
        uint32_t* cur = c->activeA.p;
        uint32_t* nxt = c->activeB.p;
        uint32_t nActive = nRows;
        uint32_t prevTarget = 0;
        float impMs = 0;
        for (uint32_t pass = 0;; ++pass) {
            const uint32_t target = adaptiveTarget(ex->minRays, maxRays, cp->adaptiveSteps, pass);
            const bool lastPass = target >= maxRays || pass >= cp->adaptiveSteps;
            const uint32_t M = target - prevTarget;
            // local proposal: the map places the near rays, the rest are far
            // rays; both parts get at least one ray (a one-ray pass is near only)
            const uint32_t Mfar = farPrior && M >= 2u
                                      ? uint32_t(std::min<long long>(M - 1u, std::max(1ll, std::llround(double(M) *
                                                                                                       c->farFraction))))
                                      : 0u;
            const uint32_t Mnear = M - Mfar;
            MapLaunch ml{c->lnw.p, 1, pass == 0 ? 1 : 0, cur, nW, Mnear, nullptr, firstSample, pass, cp->rngSeed, 0u,
                         nullptr, c->q.p, c->Q.p, c->offsets.p};
            mapKernel<<<nActive, kMapBlock, 0, c->stream>>>(ml);
            HASE_CUDA(cudaGetLastError());
            const uint32_t itemRays = std::max<uint32_t>(cp->raysPerThread ? 32u * cp->raysPerThread : kMinItemRays,
                                                         (M + kMaxItems - 1) / kMaxItems);
            const uint32_t items = (M + itemRays - 1) / itemRays;
            HASE_CUDA(cudaMemsetAsync(c->itemCounter.p, 0, sizeof(unsigned int), c->stream));
            HASE_CUDA(cudaEventRecord(c->ev[2], c->stream));
            RayLaunch rl{mv, cur, nActive, firstSample, pass, M, nW, itemRays, items, c->itemCounter.p, c->q.p,
                         c->Q.p, c->offsets.p, cp->rngSeed, 0u, c->spec.p, nLambda, ex->nearFieldSampling, C, c->pSum.p, c->pSum2.p,
                         c->pDrop.p, c->pCross.p, logOut ? c->logBuf.p : nullptr};
            if (local) {
                rl.cand = c->candTri.p;
                rl.candSorted = c->candSorted.p;
                rl.candRank = c->candRank.p;
                rl.K = K;
                rl.Mnear = Mnear;
                rl.slices = slices;
                rl.divKm = divKm;
                rl.divKs = divKs;
                rl.nearShare = float(double(Mnear) / double(M));
                rl.farShare = float(double(Mfar) / double(M));
                if (farPrior) rl.far = farView(c, slices);
            }
            const RayVariant logVariant{rayKernel<kRayBlock, kRefill, kRayMinBlocks, true>, int(kRayBlock), "log"};
            const RayVariant localLog{rayKernel<kRayBlock, kRefill, kRayMinBlocks, true, false, kWalkColumns, kWalkBeta, true>,
                                      int(kRayBlock), "local log"};
            const RayVariant& rv = local ? (logOut ? localLog : kLocalVariant) : (logOut ? logVariant : kRayVariants[variant]);
            const uint64_t totalItems = uint64_t(nActive) * items;
            void (*const kern)(RayLaunch) = walk == kWalkTable ? rv.mono : (walk == kWalkBetaNoClad ? rv.noClad : rv.kernel);
            uint32_t resident = c->variantBlocks[walk][variant];
            if (local) {  // occupancy of the local kernel itself
                int perSM = 0, sms = 0;
                HASE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kern, rv.block, 0));
                HASE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
                resident = uint32_t(std::max(1, perSM) * std::max(1, sms));
            }
            const uint32_t grid = uint32_t(std::min<uint64_t>(totalItems / (rv.block / 32) + 1, uint64_t(resident)));
            void* rayArgs[] = {&rl};
            HASE_CUDA(cudaLaunchKernel(reinterpret_cast<const void*>(kern), dim3(grid), dim3(rv.block), rayArgs, 0,
                                       c->stream));
            HASE_CUDA(cudaEventRecord(c->ev[3], c->stream));
            HASE_CUDA(cudaMemsetAsync(c->counter.p, 0, sizeof(uint32_t), c->stream));
            FinalizeLaunch fl{cur, nActive, items, M, lastPass ? 1 : 0, ex->mseThreshold, c->pSum.p, c->pSum2.p,
                              c->pDrop.p, c->pCross.p, c->accSum.p, c->accSum2.p, c->accTotal.p, c->accDrop.p,
                              c->accCross.p, c->phi.p, c->mse.p, nxt, c->counter.p};
            finalizeKernel<<<(nActive * 32 + 127) / 128, 128, 0, c->stream>>>(fl);
            HASE_CUDA(cudaGetLastError());
            res->kernelLaunches += 3;  // map + rays + finalize
            uint32_t next = 0;
            HASE_CUDA(cudaMemcpyAsync(&next, c->counter.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
            HASE_CUDA(cudaStreamSynchronize(c->stream));
            float ms = 0;
            if (pass == 0) {
                HASE_CUDA(cudaEventElapsedTime(&impMs, c->ev[0], c->ev[1]));
                res->importanceMilliseconds += impMs;
            }
            HASE_CUDA(cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]));
            res->rayMilliseconds += ms;
            res->passes = std::max(res->passes, pass + 1);
            prevTarget = target;
            if (lastPass) {
                res->unconvergedSamples += next;  // samples still above threshold at the cap
                break;
            }
            if (next == 0) break;
            if (la && pass == 0 && la->fallbackVariance > 0.0f) {
                // the plain method judges: samples whose per-ray relative
                // variance under the learned proposal exceeds the plain
                // method's restart with the importance weights
                hList.resize(next);
                hRse.resize(nRows);
                hTot.resize(nRows);
                HASE_CUDA(cudaMemcpyAsync(hList.data(), nxt, next * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
                HASE_CUDA(cudaMemcpyAsync(hRse.data(), c->mse.p, nRows * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
                HASE_CUDA(cudaMemcpyAsync(hTot.data(), c->accTotal.p, nRows * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                          c->stream));
                HASE_CUDA(cudaStreamSynchronize(c->stream));
                std::vector<uint32_t> fb;
                for (uint32_t i = 0; i < next; ++i) {
                    const uint32_t r = hList[i];
                    const double v = double(hTot[r]) * hRse[r] * hRse[r];
                    if (!std::isfinite(hRse[r]) || v > double(la->fallbackVariance)) fb.push_back(r);
                }
                if (!fb.empty()) {
                    const uint32_t nf = uint32_t(fb.size());
                    HASE_CUDA(cudaMemcpyAsync(c->rowList.p, fb.data(), nf * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                              c->stream));
                    HASE_CUDA(cudaEventRecord(c->ev[2], c->stream));
                    il.rowList = c->rowList.p;
                    launchImportanceRows(nf);
                    il.rowList = nullptr;
                    HASE_CUDA(cudaGetLastError());
                    HASE_CUDA(cudaEventRecord(c->ev[3], c->stream));
                    MapLaunch rq{c->lnw.p, 1, 1, c->rowList.p, nW, 1u, nullptr, firstSample, 0u, cp->rngSeed, 0u,
                                 nullptr, c->q.p, c->Q.p, c->offsets.p};
                    mapKernel<<<nf, kMapBlock, 0, c->stream>>>(rq);
                    resetRowsKernel<<<(nf + 255) / 256, 256, 0, c->stream>>>(c->rowList.p, nf, c->accSum.p,
                                                                             c->accSum2.p, c->accTotal.p,
                                                                             c->accDrop.p, c->accCross.p);
                    HASE_CUDA(cudaGetLastError());
                    res->kernelLaunches += 3;
                    HASE_CUDA(cudaStreamSynchronize(c->stream));
                    float fbMs = 0.0f;
                    HASE_CUDA(cudaEventElapsedTime(&fbMs, c->ev[2], c->ev[3]));
                    res->importanceMilliseconds += fbMs;
                    la->fallbackSamples += nf;
                }
            }
            std::swap(cur, nxt);
            nActive = next;
        }
        HASE_CUDA(cudaEventRecord(c->ev[3], c->stream));
        HASE_CUDA(cudaMemcpyAsync(hPhi.data(), c->phi.p, nRows * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
        HASE_CUDA(cudaMemcpyAsync(hMse.data(), c->mse.p, nRows * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        HASE_CUDA(cudaMemcpyAsync(hTotal.data(), c->accTotal.p, nRows * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
        HASE_CUDA(cudaMemcpyAsync(hDrop.data(), c->accDrop.p, nRows * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
        HASE_CUDA(cudaMemcpyAsync(hCross.data(), c->accCross.p, nRows * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
        if (logOut)
            HASE_CUDA(cudaMemcpyAsync(logOut + size_t(b0) * nW, c->logBuf.p, size_t(nRows) * nW * sizeof(float),
                                      cudaMemcpyDeviceToHost, c->stream));
        HASE_CUDA(cudaStreamSynchronize(c->stream));
        float total = 0;
        HASE_CUDA(cudaEventElapsedTime(&total, c->ev[0], c->ev[3]));
        res->totalMilliseconds += total;
        for (uint32_t i = 0; i < nRows; ++i) {
            const uint32_t o = b0 + i, s = firstSample + i;
            if (res->phiAse) res->phiAse[o] = hPhi[i];
            if (res->relativeStandardError) res->relativeStandardError[o] = hMse[i];
            if (res->standardError) res->standardError[o] = hMse[i] * double(hPhi[i]);
            if (res->totalRays) res->totalRays[o] = hTotal[i];
            if (res->droppedRays) res->droppedRays[o] = hDrop[i];
            if (res->dndtAse) {
                const double sA = nLambda == 1 ? c->sigmaA[0] : maxSA, sE = nLambda == 1 ? c->sigmaE[0] : maxSE;
                const double bc = c->betaCells.empty() ? 0.0 : c->betaCells[s];
                res->dndtAse[o] = (bc * (sE + sA) - sA) * double(hPhi[i]);
            }
            res->raysTraced += hTotal[i];
            res->crossings += hCross[i];
            droppedTotal += hDrop[i];
        }
    }
    if (droppedTotal) {
        fail(HASE_DROPPED_RAYS, "%llu rays could not be walked", (unsigned long long)droppedTotal);
        return HASE_DROPPED_RAYS;
    }
    if (res->unconvergedSamples) {
        fail(HASE_NOT_CONVERGED, "%u samples above the threshold at maxRays", res->unconvergedSamples);
        return HASE_NOT_CONVERGED;
    }
    return HASE_OK;
}


hase_status hase_calc_phi_ase(hase_context* c, const hase_experiment_desc* ex, const hase_compute_desc* cp,
                              hase_result* res) {
    return calcCore(c, ex, cp, res, nullptr, nullptr);
}

}  // extern "C"

namespace {

// The phi-ASE source of one step of the time loop: fills phiPrism (device,
// [P] FP32, the ASE flux per prism), adds its device time, rays and the mean
// phi it reports; returns the solve's status (warnings allowed).
struct AseSource {
    virtual ~AseSource() = default;
    virtual hase_status solve(uint32_t step, float* phiPrism, double& ms, uint64_t& rays, double& meanPhi) = 0;
};

// Time-stepped rate equations (include/core/timeSteppedSimulation.hpp:132-617,
// include/kernels/derivativeComposition.hpp:27-93): per step the ASE source,
// then the pump by exact column Beer-Lambert and the frozen-ASE RK4 / Euler
// update of beta on the device.  sA / sE are the ASE cross sections of the
// depletion term.
hase_status simulateCore(hase_context* c, double sA, double sE, AseSource& source, const hase_pump_desc* pd,
                         const hase_time_desc* td, hase_time_result* res, std::vector<double>& betaHost) {
    if (!c || !pd || !td || !res) return fail(HASE_INVALID_ARGUMENT, "null argument");
    if (!(td->timeStep > 0.0) || td->steps == 0) return fail(HASE_INVALID_ARGUMENT, "timeStep and steps must be positive");
    if (td->integrator >= kNumIntegrators) return fail(HASE_INVALID_ARGUMENT, "integrator must be 0 .. 6");
    if (td->aseSteps > td->steps) return fail(HASE_INVALID_ARGUMENT, "aseSteps > steps");
    if (!(pd->radius > 0.0) || !(pd->exponent > 0.0) || !(pd->wavelength > 0.0) || !(pd->peakIntensity >= 0.0) ||
        !(pd->sigmaA >= 0.0) || !(pd->sigmaE >= 0.0))
        return fail(HASE_INVALID_ARGUMENT, "pump parameters must be positive (intensity and cross sections >= 0)");
    HASE_TRY(setDevice(c));
    const uint32_t P = c->P, T = c->T;
    std::vector<uint8_t> clad(P, 0);
    if (!c->cladTypes.empty())
        for (uint32_t p = 0; p < P; ++p) clad[p] = c->cladTypes[p % T] == c->cladNumber ? 1 : 0;
    DevBuf<double> beta0, stage, nextB, kb, rate, absorbed;
    DevBuf<float> phiP, area;
    DevBuf<uint8_t> dclad;
    HASE_CUDA(beta0.ensure(P));
    HASE_CUDA(stage.ensure(P));
    HASE_CUDA(nextB.ensure(P));
    HASE_CUDA(kb.ensure(4 * size_t(P)));
    HASE_CUDA(rate.ensure(P));
    HASE_CUDA(absorbed.ensure(1));
    HASE_CUDA(phiP.ensure(P));
    HASE_CUDA(area.ensure(T));
    HASE_CUDA(dclad.ensure(P));
    HASE_CUDA(cudaMemcpyAsync(beta0.p, c->hBeta.data(), P * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    HASE_CUDA(cudaMemcpyAsync(area.p, c->hArea.data(), T * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    HASE_CUDA(cudaMemcpyAsync(dclad.p, clad.data(), P, cudaMemcpyHostToDevice, c->stream));
    const double photon = 6.62607015e-34 * 2.99792458e8 / pd->wavelength;  // J
    PumpLaunch pl{};
    pl.centroid = c->centroid.p;
    pl.clad = dclad.p;
    pl.rate = rate.p;
    pl.area = area.p;
    pl.T = T;
    pl.layers = c->layers;
    pl.h = c->h;
    pl.nTot = c->nTot;
    pl.sA = pd->sigmaA;
    pl.sE = pd->sigmaE;
    pl.cladAbs = c->cladAbs;
    pl.flux0 = pd->peakIntensity / photon;
    pl.radius = pd->radius;
    pl.expo = pd->exponent;
    pl.cx = pd->centerX;
    pl.cy = pd->centerY;
    pl.retro = pd->retroreflect ? 1 : 0;
    double incident = 0.0;  // photons / s entering the bottom surface
    for (uint32_t t = 0; t < T; ++t) {
        const double dx = c->hCentroid[t].x - pd->centerX, dy = c->hCentroid[t].y - pd->centerY;
        incident += pl.flux0 * std::exp(-std::pow(std::sqrt(dx * dx + dy * dy) / pd->radius, pd->exponent)) *
                    c->hArea[t];
    }
    betaHost = c->hBeta;
    res->aseMilliseconds = res->pumpMilliseconds = res->totalMilliseconds = 0.0;
    res->raysTraced = 0;
    res->fallbackSamples = 0;
    auto meanGain = [&](const std::vector<double>& b) {
        double sum = 0.0;
        uint32_t n = 0;
        for (uint32_t p = 0; p < P; ++p)
            if (!clad[p]) {
                sum += b[p];
                ++n;
            }
        return n ? sum / n : 0.0;
    };
    if (res->meanBeta) res->meanBeta[0] = meanGain(c->hBeta);
    uint32_t solveIndex = 0;  // phi-ASE solves so far (the index of phiHistory)
    const uint32_t blocksP = (P + 255) / 256, blocksT = (T + 255) / 256;
    const double dt = td->timeStep;
    const uint32_t method = td->integrator;
    const uint32_t implicitIterations = std::max(1u, td->implicitIterations ? td->implicitIterations : 8u);
    hase_status worst = HASE_OK;
    // device timing of the pump / derivative / update kernels: one event pair
    // per group of launches between phi-ASE solves, read after each step
    std::vector<cudaEvent_t> evPool;
    struct EvPool {
        std::vector<cudaEvent_t>& v;
        ~EvPool() {
            for (cudaEvent_t e : v) cudaEventDestroy(e);
        }
    } evPoolOwner{evPool};
    size_t evUsed = 0;
    auto nextEvent = [&](cudaEvent_t& e) -> hase_status {
        if (evUsed == evPool.size()) {
            cudaEvent_t n = nullptr;
            HASE_CUDA(cudaEventCreate(&n));
            evPool.push_back(n);
        }
        e = evPool[evUsed++];
        return HASE_OK;
    };
    // tables of the walks (device) and host copies of beta (the learned
    // proposal's features, the forward twin) set to the state `b`
    auto setState = [&](const double* b) -> hase_status {
        betaToTablesKernel<<<blocksP, 256, 0, c->stream>>>(b, dclad.p, c->gainBeta.p, c->srcBeta.p, P);
        HASE_CUDA(cudaGetLastError());
        HASE_CUDA(cudaMemcpyAsync(betaHost.data(), b, P * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        HASE_CUDA(cudaStreamSynchronize(c->stream));
        c->hBeta = betaHost;
        for (uint32_t p = 0; p < P; ++p) c->hGainBeta[p] = clad[p] ? NAN : float(betaHost[p]);
        ++c->betaVersion;  // the learned proposal's feature grid follows the new beta
        return HASE_OK;
    };
    for (uint32_t step = 0; step < td->steps; ++step) {
        const bool ase = step < td->aseSteps, pumpOn = step < td->pumpSteps;
        bool firstSolve = true, firstPump = true, tablesAtStart = true;
        evUsed = 0;
        if (res->meanPhi) res->meanPhi[step] = 0.0;
        HASE_CUDA(cudaMemsetAsync(absorbed.p, 0, sizeof(double), c->stream));
        // phi-ASE of the state `b` (phiP), solved when `refresh` (otherwise the
        // step's last solve stays in use, the frozen-ASE stages)
        auto solveAt = [&](const double* b, bool refresh) -> hase_status {
            if (!ase || !refresh) return HASE_OK;
            if (b != beta0.p || !tablesAtStart) {
                HASE_TRY(setState(b));
                tablesAtStart = b == beta0.p;
            }
            double ms = 0.0, mp = 0.0;
            uint64_t rays = 0;
            const hase_status st = source.solve(solveIndex, phiP.p, ms, rays, mp);
            if (st != HASE_OK && st != HASE_NOT_CONVERGED && st != HASE_DROPPED_RAYS) return st;
            if (st != HASE_OK && worst == HASE_OK) worst = st;
            ++solveIndex;
            res->aseMilliseconds += ms;
            res->totalMilliseconds += ms;
            res->raysTraced += rays;
            if (firstSolve && res->meanPhi) res->meanPhi[step] = mp;
            firstSolve = false;
            return HASE_OK;
        };
        // pump rate of the state `b` (the absorbed power of the step's first evaluation)
        auto pumpAt = [&](const double* b) -> hase_status {
            HASE_CUDA(cudaMemsetAsync(rate.p, 0, P * sizeof(double), c->stream));
            if (pumpOn) {
                pl.beta = b;
                pl.absorbed = firstPump ? absorbed.p : nullptr;
                pumpColumnKernel<<<blocksT, 256, 0, c->stream>>>(pl);
            }
            firstPump = false;
            return HASE_OK;
        };
        // k[idx] = derivative at `b`, phi-ASE re-solved there when `refresh`
        auto evaluate = [&](const double* b, uint32_t idx, bool refresh) -> hase_status {
            HASE_TRY(solveAt(b, refresh));
            cudaEvent_t ea, eb;
            HASE_TRY(nextEvent(ea));
            HASE_TRY(nextEvent(eb));
            HASE_CUDA(cudaEventRecord(ea, c->stream));
            HASE_TRY(pumpAt(b));
            rateDerivativeKernel<<<blocksP, 256, 0, c->stream>>>(b, rate.p, ase ? phiP.p : nullptr, dclad.p,
                                                                kb.p + size_t(idx) * P, P, sA, sE, c->tau);
            HASE_CUDA(cudaGetLastError());
            HASE_CUDA(cudaEventRecord(eb, c->stream));
            return HASE_OK;
        };
        auto axpy = [&](const double* base, uint32_t idx, double a, double* out) -> hase_status {
            rateAxpyKernel<<<blocksP, 256, 0, c->stream>>>(base, kb.p + size_t(idx) * P, a, out, P);
            return cudaGetLastError() == cudaSuccess ? HASE_OK : fail(HASE_CUDA_ERROR, "stage update failed");
        };
        // the step, in the reference's stage order (include/core/timeSteppedSimulation.hpp:321-415)
        switch (method) {
            case kExplicitEuler:
                HASE_TRY(evaluate(beta0.p, 0, true));
                break;
            case kHeun:
                HASE_TRY(evaluate(beta0.p, 0, true));
                HASE_TRY(axpy(beta0.p, 0, dt, stage.p));
                HASE_TRY(evaluate(stage.p, 1, true));
                break;
            case kMidpoint:
                HASE_TRY(evaluate(beta0.p, 0, true));
                HASE_TRY(axpy(beta0.p, 0, 0.5 * dt, stage.p));
                HASE_TRY(evaluate(stage.p, 1, true));
                break;
            case kFrozenRk4:
            case kRk4: {
                const bool re = method == kRk4;
                HASE_TRY(evaluate(beta0.p, 0, true));
                HASE_TRY(axpy(beta0.p, 0, 0.5 * dt, stage.p));
                HASE_TRY(evaluate(stage.p, 1, re));
                HASE_TRY(axpy(beta0.p, 1, 0.5 * dt, nextB.p));
                HASE_TRY(evaluate(nextB.p, 2, re));
                HASE_TRY(axpy(beta0.p, 2, dt, stage.p));
                HASE_TRY(evaluate(stage.p, 3, re));
                break;
            }
            case kImplicitEuler: {
                // stage = beta; repeat: stage = beta + dt k(stage), phi-ASE re-solved each time
                const double* cur = beta0.p;
                for (uint32_t it = 0; it < implicitIterations; ++it) {
                    HASE_TRY(evaluate(cur, 0, true));
                    double* out = (it % 2 == 0) ? stage.p : nextB.p;
                    HASE_TRY(axpy(beta0.p, 0, dt, out));
                    cur = out;
                }
                break;
            }
            default:  // kExpEuler
                HASE_TRY(solveAt(beta0.p, true));
                break;
        }
        cudaEvent_t ea, eb;
        HASE_TRY(nextEvent(ea));
        HASE_TRY(nextEvent(eb));
        HASE_CUDA(cudaEventRecord(ea, c->stream));
        if (method == kExpEuler) {
            HASE_TRY(pumpAt(beta0.p));
            rateExpEulerKernel<<<blocksP, 256, 0, c->stream>>>(beta0.p, rate.p, ase ? phiP.p : nullptr, dclad.p,
                                                              nextB.p, P, sA, sE, c->tau, dt);
        } else {
            rateCombineKernel<<<blocksP, 256, 0, c->stream>>>(beta0.p, kb.p, method, dt, nextB.p, P);
        }
        HASE_CUDA(cudaMemcpyAsync(beta0.p, nextB.p, P * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        betaToTablesKernel<<<blocksP, 256, 0, c->stream>>>(beta0.p, dclad.p, c->gainBeta.p, c->srcBeta.p, P);
        HASE_CUDA(cudaGetLastError());
        HASE_CUDA(cudaEventRecord(eb, c->stream));
        double abs = 0.0;
        HASE_CUDA(cudaMemcpyAsync(&abs, absorbed.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        HASE_CUDA(cudaMemcpyAsync(betaHost.data(), beta0.p, P * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        HASE_CUDA(cudaStreamSynchronize(c->stream));
        for (size_t e = 0; e + 1 < evUsed; e += 2) {
            float ms = 0.0f;
            HASE_CUDA(cudaEventElapsedTime(&ms, evPool[e], evPool[e + 1]));
            res->pumpMilliseconds += ms;
            res->totalMilliseconds += ms;
        }
        if (res->pumpAbsorbed) res->pumpAbsorbed[step] = pumpOn && incident > 0.0 ? abs / incident : 0.0;
        // host copies the next solve's features read
        c->hBeta = betaHost;
        for (uint32_t p = 0; p < P; ++p) c->hGainBeta[p] = clad[p] ? NAN : float(betaHost[p]);
        ++c->betaVersion;  // the learned proposal's feature grid follows the new beta
        if (res->meanBeta) res->meanBeta[step + 1] = meanGain(betaHost);
    }
    if (res->betaVolume) std::copy(betaHost.begin(), betaHost.end(), res->betaVolume);
    if (worst != HASE_OK) return fail(worst, "a phi-ASE solve of the time loop ended with a warning");
    return HASE_OK;
}

// ASE from the backward solve over every sample point (importance weights or
// the learned proposal); a prism's phi is the mean of its six vertices.
struct BackwardAse final : AseSource {
    hase_context* c;
    const hase_experiment_desc* ex;
    hase_compute_desc all;
    LearnedArgs la;
    bool learned;
    float* phiHistory;
    uint32_t fallbackSamples = 0;
    std::vector<float> phiHost;
    DevBuf<float> phiS;
    hase_status solve(uint32_t step, float* phiPrism, double& ms, uint64_t& rays, double& meanPhi) override {
        const uint32_t S = c->Np * c->L;
        phiHost.resize(S);
        HASE_CUDA(phiS.ensure(S));
        hase_result r{};
        r.phiAse = phiHost.data();
        const hase_status st = calcCore(c, ex, &all, &r, learned ? &la : nullptr, nullptr);
        if (st != HASE_OK && st != HASE_NOT_CONVERGED && st != HASE_DROPPED_RAYS) return st;
        ms = r.totalMilliseconds;
        rays = r.raysTraced;
        if (learned) fallbackSamples += la.fallbackSamples;
        double mp = 0.0;
        for (uint32_t k = 0; k < S; ++k) mp += phiHost[k];
        meanPhi = mp / S;
        if (phiHistory) std::copy(phiHost.begin(), phiHost.end(), phiHistory + size_t(step) * S);
        HASE_CUDA(cudaMemcpyAsync(phiS.p, phiHost.data(), S * sizeof(float), cudaMemcpyHostToDevice, c->stream));
        phiPrismKernel<<<(c->P + 255) / 256, 256, 0, c->stream>>>(c->verts.p, phiS.p, phiPrism, c->T, c->layers,
                                                                 c->Np);
        HASE_CUDA(cudaGetLastError());
        return st;
    }
};

// ASE from the forward method on the Tet4 twin (cell 3p + k belongs to prism
// p): the prisms' beta go to their cells, one forward solve, a prism's phi is
// the volume-weighted mean of its three cells.
struct ForwardAse final : AseSource {
    hase_context* c;
    hase_tet_context* twin;
    const hase_forward_desc* fw;
    float* phiHistory;
    const std::vector<double>* beta;  // the loop's current prism beta (host)
    std::vector<double> vol, betaCells, rseCells;
    std::vector<float> phiCells, phiHost;
    std::vector<uint8_t> clad;
    uint32_t srmStatus = 0;
    hase_status solve(uint32_t step, float* phiPrism, double& ms, uint64_t& rays, double& meanPhi) override {
        const uint32_t P = c->P;
        betaCells.resize(3 * size_t(P));
        for (uint32_t p = 0; p < P; ++p)
            for (int k = 0; k < 3; ++k) betaCells[3 * size_t(p) + k] = (*beta)[p];
        HASE_TRY(hase_tet_context_update_beta(twin, betaCells.data()));
        phiCells.resize(3 * size_t(P));
        hase_forward_result r{};
        r.phiAse = phiCells.data();
        const hase_status st = hase_tet_calc_phi_ase(twin, fw, &r);
        if (st != HASE_OK && st != HASE_NOT_CONVERGED && st != HASE_DROPPED_RAYS) return st;
        ms = r.totalMilliseconds;
        rays = r.raysTraced;
        srmStatus = std::max(srmStatus, r.srmStatus == 3 ? 4u : r.srmStatus == 4 ? 3u : r.srmStatus);
        phiHost.resize(P);
        double mp = 0.0;
        uint32_t n = 0;
        for (uint32_t p = 0; p < P; ++p) {
            double num = 0.0, den = 0.0;
            for (int k = 0; k < 3; ++k) {
                num += vol[3 * size_t(p) + k] * double(phiCells[3 * size_t(p) + k]);
                den += vol[3 * size_t(p) + k];
            }
            phiHost[p] = float(den > 0.0 ? num / den : 0.0);
            if (!clad[p]) {
                mp += phiHost[p];
                ++n;
            }
        }
        meanPhi = n ? mp / n : 0.0;
        if (phiHistory) std::copy(phiHost.begin(), phiHost.end(), phiHistory + size_t(step) * P);
        HASE_CUDA(cudaMemcpyAsync(phiPrism, phiHost.data(), P * sizeof(float), cudaMemcpyHostToDevice, c->stream));
        return st;
    }
};

}  // namespace

extern "C" {

hase_status hase_simulate(hase_context* c, hase_proposal* net, float fallbackVariance,
                          const hase_experiment_desc* ex, const hase_compute_desc* cp, const hase_pump_desc* pd,
                          const hase_time_desc* td, hase_time_result* res) {
    if (!c || !ex || !cp || !pd || !td || !res) return fail(HASE_INVALID_ARGUMENT, "null argument");
    if (!(fallbackVariance >= 0.0f)) return fail(HASE_INVALID_ARGUMENT, "fallbackVariance must be >= 0");
    const uint32_t nL = ex->monochromatic ? 1u : uint32_t(c->sigmaA.size());
    double sA = c->sigmaA[0], sE = c->sigmaE[0];
    for (uint32_t l = 1; l < nL; ++l) {
        sA = std::max(sA, c->sigmaA[l]);
        sE = std::max(sE, c->sigmaE[l]);
    }
    BackwardAse src;
    src.c = c;
    src.ex = ex;
    src.all = *cp;
    src.all.minSample = 0;
    src.all.maxSample = UINT32_MAX;
    src.la = LearnedArgs{net, 0.1f, fallbackVariance, 0u};
    src.learned = net != nullptr;
    src.phiHistory = res->phiHistory;
    std::vector<double> betaHost;
    const hase_status st = simulateCore(c, sA, sE, src, pd, td, res, betaHost);
    res->fallbackSamples = src.fallbackSamples;
    return st;
}

hase_status hase_simulate_forward(hase_context* c, hase_tet_context* twin, const hase_forward_desc* fw,
                                  const hase_pump_desc* pd, const hase_time_desc* td, hase_time_result* res) {
    if (!c || !twin || !fw || !pd || !td || !res) return fail(HASE_INVALID_ARGUMENT, "null argument");
    const size_t C = 3 * size_t(c->P);
    ForwardAse src;
    uint32_t cells = 0, points = 0;
    HASE_TRY(hase_tet_context_info(twin, &cells, &points));
    if (cells != C)
        return fail(HASE_INVALID_ARGUMENT, "the Tet4 twin has %u cells, the prism mesh needs 3 x %u", cells, c->P);
    src.vol.resize(C);
    HASE_TRY(hase_tet_tables(twin, nullptr, nullptr, nullptr, src.vol.data()));
    const uint32_t nL = fw->monochromatic ? 1u : uint32_t(c->sigmaA.size());
    double sA = c->sigmaA[0], sE = c->sigmaE[0];
    for (uint32_t l = 1; l < nL; ++l) {
        sA = std::max(sA, c->sigmaA[l]);
        sE = std::max(sE, c->sigmaE[l]);
    }
    src.c = c;
    src.twin = twin;
    src.fw = fw;
    src.phiHistory = res->phiHistory;
    src.clad.assign(c->P, 0);
    if (!c->cladTypes.empty())
        for (uint32_t p = 0; p < c->P; ++p) src.clad[p] = c->cladTypes[p % c->T] == c->cladNumber ? 1 : 0;
    std::vector<double> betaHost;
    src.beta = &betaHost;
    res->fallbackSamples = 0;
    return simulateCore(c, sA, sE, src, pd, td, res, betaHost);
}

hase_status hase_calc_phi_ase_learned(hase_context* c, hase_proposal* net, const hase_experiment_desc* ex,
                                      const hase_compute_desc* cp, hase_learned_desc* learned, hase_result* res) {
    if (!net || !learned) return fail(HASE_INVALID_ARGUMENT, "null argument");
    if (!(learned->mixture >= 0.0f) || learned->mixture >= 1.0f)
        return fail(HASE_INVALID_ARGUMENT, "mixture must be in [0, 1)");
    if (!(learned->fallbackVariance >= 0.0f)) return fail(HASE_INVALID_ARGUMENT, "fallbackVariance must be >= 0");
    LearnedArgs la{net, learned->mixture > 0.0f ? learned->mixture : 0.1f, learned->fallbackVariance, 0u};
    const hase_status st = calcCore(c, ex, cp, res, &la, nullptr);
    learned->fallbackSamples = la.fallbackSamples;
    int err = 0;
    if (cudaMemcpy(&err, net->error.p, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess && err)
        return fail(HASE_DEVICE_TIMEOUT, "a tensor-core wait of the proposal network timed out");
    return st;
}

hase_status hase_log_contributions(hase_context* c, const hase_experiment_desc* ex, const hase_compute_desc* cp,
                                   float* contributions, hase_result* res) {
    if (!contributions) return fail(HASE_INVALID_ARGUMENT, "null argument");
    hase_result local{};
    return calcCore(c, ex, cp, res ? res : &local, nullptr, contributions);
}

hase_status hase_proposal_features(hase_context* c, uint32_t firstSample, uint32_t count, uint32_t useReflections,
                                   uint32_t monochromatic, float* features) {
    if (!c || !features) return fail(HASE_INVALID_ARGUMENT, "null argument");
    if (count == 0) return HASE_OK;
    if (uint64_t(firstSample) + count > uint64_t(c->Np) * c->L)
        return fail(HASE_INVALID_ARGUMENT, "sample range outside the mesh");
    HASE_TRY(setDevice(c));
    if (c->localK) HASE_TRY(prepareLocal(c));
    const uint32_t nW = rowEntries(c, useReflections ? 5u : 1u);
    const uint32_t nL = monochromatic ? 1u : uint32_t(c->sigmaA.size());
    double A = 0.0, B = 0.0;
    for (uint32_t l = 0; l < nL; ++l) {
        A += c->nTot * (c->sigmaE[l] + c->sigmaA[l]) / nL;
        B += c->nTot * c->sigmaA[l] / nL;
    }
    ProposalView pv{};
    HASE_TRY(buildProposalView(c, A, B, pv));
    pv.firstSample = firstSample;
    pv.nW = nW;
    localFields(c, pv);
    const size_t n = size_t(count) * nW * kFeat;
    DevBuf<float> out;
    HASE_CUDA(out.ensure(n));
    ProposalLaunch pl{pv, nullptr, nullptr, nullptr, nullptr, out.p, count, nullptr};
    const uint64_t pairs = uint64_t(count) * nW;
    featureKernel<<<uint32_t((pairs + 255) / 256), 256, 0, c->stream>>>(pl);
    HASE_CUDA(cudaGetLastError());
    HASE_CUDA(cudaMemcpyAsync(features, out.p, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    HASE_CUDA(cudaStreamSynchronize(c->stream));
    return HASE_OK;
}

hase_status hase_importance_weights(hase_context* c, uint32_t firstSample, uint32_t count, uint32_t useReflections,
                                    float* weights) {
    if (!c || !weights || count == 0) return fail(HASE_INVALID_ARGUMENT, "bad argument");
    if (uint64_t(firstSample) + count > uint64_t(c->Np) * c->L) return fail(HASE_INVALID_ARGUMENT, "sample range");
    HASE_TRY(setDevice(c));
    if (c->localK) HASE_TRY(prepareLocal(c));
    const uint32_t slices = useReflections ? 5u : 1u, nW = rowEntries(c, slices);
    double meanA = 0, meanB = 0;
    const uint32_t n = uint32_t(c->sigmaA.size());
    for (uint32_t l = 0; l < n; ++l) {
        meanA += c->nTot * (c->sigmaE[l] + c->sigmaA[l]) / n;
        meanB += c->nTot * c->sigmaA[l] / n;
    }
    DevBuf<float> lnw, w;
    DevBuf<uint32_t> q, off;
    DevBuf<unsigned long long> Q;
    HASE_CUDA(lnw.ensure(size_t(count) * nW));
    HASE_CUDA(w.ensure(size_t(count) * nW));
    HASE_CUDA(q.ensure(size_t(count) * nW));
    HASE_CUDA(off.ensure(size_t(count) * (nW + 1)));
    HASE_CUDA(Q.ensure(count));
    ImportanceLaunch il{c->view(), firstSample, slices, nW, float(meanA), float(meanB), lnw.p};
    localFields(c, il);
    HASE_CUDA(launchImportance(0, il, c->layers, c->T, count, c->stream));
    MapLaunch ml{lnw.p, 1, 1, nullptr, nW, 1u, nullptr, firstSample, 0u, 0u, 0u, w.p, q.p, Q.p, off.p};
    mapKernel<<<count, kMapBlock, 0, c->stream>>>(ml);
    HASE_CUDA(cudaGetLastError());
    HASE_CUDA(cudaMemcpyAsync(weights, w.p, size_t(count) * nW * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    HASE_CUDA(cudaStreamSynchronize(c->stream));
    return HASE_OK;
}

hase_status hase_grid_weights(hase_context* c, uint32_t firstSample, uint32_t count, uint32_t useReflections,
                              uint32_t monochromatic, float* weights) {
    if (!c || !weights || count == 0) return fail(HASE_INVALID_ARGUMENT, "bad argument");
    if (uint64_t(firstSample) + count > uint64_t(c->Np) * c->L) return fail(HASE_INVALID_ARGUMENT, "sample range");
    HASE_TRY(setDevice(c));
    if (c->localK) HASE_TRY(prepareLocal(c));
    const uint32_t slices = useReflections ? 5u : 1u, nW = rowEntries(c, slices);
    const uint32_t nL = monochromatic ? 1u : uint32_t(c->sigmaA.size());
    double meanA = 0, meanB = 0;
    for (uint32_t l = 0; l < nL; ++l) {
        meanA += c->nTot * (c->sigmaE[l] + c->sigmaA[l]) / nL;
        meanB += c->nTot * c->sigmaA[l] / nL;
    }
    ProposalView pv{};
    HASE_TRY(cachedProposalView(c, meanA, meanB, pv));
    pv.firstSample = firstSample;
    pv.nW = nW;
    localFields(c, pv);
    DevBuf<float> lnw, w;
    DevBuf<uint32_t> q, off;
    DevBuf<unsigned long long> Q;
    HASE_CUDA(lnw.ensure(size_t(count) * nW));
    HASE_CUDA(w.ensure(size_t(count) * nW));
    HASE_CUDA(q.ensure(size_t(count) * nW));
    HASE_CUDA(off.ensure(size_t(count) * (nW + 1)));
    HASE_CUDA(Q.ensure(count));
    const ProposalLaunch gl{pv, nullptr, nullptr, lnw.p, nullptr, nullptr, count, nullptr};
    HASE_CUDA(launchGridWeights(gl, c->stream));
    MapLaunch ml{lnw.p, 1, 1, nullptr, nW, 1u, nullptr, firstSample, 0u, 0u, 0u, w.p, q.p, Q.p, off.p};
    mapKernel<<<count, kMapBlock, 0, c->stream>>>(ml);
    HASE_CUDA(cudaGetLastError());
    HASE_CUDA(cudaMemcpyAsync(weights, w.p, size_t(count) * nW * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    HASE_CUDA(cudaStreamSynchronize(c->stream));
    return HASE_OK;
}

hase_status hase_importance_crossings(hase_context* c, uint32_t firstSample, uint32_t count, uint32_t useReflections,
                                      uint64_t* crossings) {
    if (!c || !crossings || count == 0) return fail(HASE_INVALID_ARGUMENT, "bad argument");
    if (uint64_t(firstSample) + count > uint64_t(c->Np) * c->L) return fail(HASE_INVALID_ARGUMENT, "sample range");
    HASE_TRY(setDevice(c));
    if (c->localK) HASE_TRY(prepareLocal(c));
    const uint32_t slices = useReflections ? 5u : 1u, nW = rowEntries(c, slices);
    DevBuf<float> lnw;
    DevBuf<unsigned long long> n;
    HASE_CUDA(lnw.ensure(size_t(count) * nW));
    HASE_CUDA(n.ensure(1));
    HASE_CUDA(cudaMemsetAsync(n.p, 0, sizeof(unsigned long long), c->stream));
    ImportanceLaunch il{c->view(), firstSample, slices, nW, 0.0f, 0.0f, lnw.p};
    localFields(c, il);
    il.crossings = n.p;
    HASE_CUDA(launchImportance(0, il, c->layers, c->T, count, c->stream, false, true));
    unsigned long long h = 0;
    HASE_CUDA(cudaMemcpyAsync(&h, n.p, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    HASE_CUDA(cudaStreamSynchronize(c->stream));
    *crossings = h;
    return HASE_OK;
}

hase_status hase_learned_weights(hase_context* c, hase_proposal* net, uint32_t firstSample, uint32_t count,
                                uint32_t useReflections, uint32_t monochromatic, float mixture, float* weights) {
    if (!c || !net || !weights || count == 0) return fail(HASE_INVALID_ARGUMENT, "bad argument");
    if (uint64_t(firstSample) + count > uint64_t(c->Np) * c->L) return fail(HASE_INVALID_ARGUMENT, "sample range");
    if (!(mixture >= 0.0f) || mixture >= 1.0f) return fail(HASE_INVALID_ARGUMENT, "mixture must be in [0, 1)");
    if (net->device != c->device)
        return fail(HASE_INVALID_ARGUMENT, "the proposal network and the context are on different devices");
    HASE_TRY(setDevice(c));
    if (c->localK) HASE_TRY(prepareLocal(c));
    const uint32_t slices = useReflections ? 5u : 1u, nW = rowEntries(c, slices);
    // the spectral average of calcCore: over the solve's wavelengths
    const uint32_t nL = monochromatic ? 1u : uint32_t(c->sigmaA.size());
    double meanA = 0, meanB = 0;
    for (uint32_t l = 0; l < nL; ++l) {
        meanA += c->nTot * (c->sigmaE[l] + c->sigmaA[l]) / nL;
        meanB += c->nTot * c->sigmaA[l] / nL;
    }
    ProposalView pv{};
    HASE_TRY(cachedProposalView(c, meanA, meanB, pv));
    pv.firstSample = firstSample;
    pv.nW = nW;
    localFields(c, pv);
    DevBuf<float> lnw, prior, w;
    DevBuf<uint32_t> q, off;
    DevBuf<unsigned long long> Q;
    HASE_CUDA(lnw.ensure(size_t(count) * nW));
    HASE_CUDA(prior.ensure(size_t(count) * nW));
    HASE_CUDA(w.ensure(size_t(count) * nW));
    HASE_CUDA(q.ensure(size_t(count) * nW));
    HASE_CUDA(off.ensure(size_t(count) * (nW + 1)));
    HASE_CUDA(Q.ensure(count));
    HASE_CUDA(cudaFuncSetAttribute(proposalKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemBytes)));
    int sms = 0;
    HASE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    ProposalLaunch pl{pv, net->wimg.p, net->vec.p, lnw.p, prior.p, nullptr, count, net->error.p};
    const uint64_t tiles = (uint64_t(count) * nW + kTile - 1) / kTile;
    proposalKernel<<<uint32_t(std::min<uint64_t>(tiles, uint64_t(std::max(1, sms)) * kMlpBlocksPerSM)), kTile,
                     kSmemBytes, c->stream>>>(pl);
    HASE_CUDA(cudaGetLastError());
    mixtureKernel<<<count, 1024, 0, c->stream>>>(nW, lnw.p, prior.p, mixture > 0.0f ? mixture : 0.1f);
    HASE_CUDA(cudaGetLastError());
    MapLaunch ml{lnw.p, 1, 1, nullptr, nW, 1u, nullptr, firstSample, 0u, 0u, 0u, w.p, q.p, Q.p, off.p};
    mapKernel<<<count, kMapBlock, 0, c->stream>>>(ml);
    HASE_CUDA(cudaGetLastError());
    HASE_CUDA(cudaMemcpyAsync(weights, w.p, size_t(count) * nW * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    HASE_CUDA(cudaStreamSynchronize(c->stream));
    int err = 0;
    HASE_CUDA(cudaMemcpy(&err, net->error.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return fail(HASE_DEVICE_TIMEOUT, "a tensor-core wait of the proposal network timed out");
    return HASE_OK;
}

hase_status hase_ray_map(uint32_t rows, uint32_t n, const float* weights, uint32_t rays, const uint32_t* phases,
                         uint32_t* q, uint32_t* offsets, uint64_t* Qout) {
    if (!weights || !phases || !q || !offsets || !Qout || rows == 0 || n == 0)
        return fail(HASE_INVALID_ARGUMENT, "bad argument");
    for (size_t i = 0; i < size_t(rows) * n; ++i)
        if (!(weights[i] >= 0.0f) || std::isinf(weights[i]))
            return fail(HASE_INVALID_ARGUMENT, "weights must be finite and non-negative");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(HASE_NO_DEVICE, "no CUDA device available");
    }
    DevBuf<float> w;
    DevBuf<uint32_t> dq, doff, dph;
    DevBuf<unsigned long long> dQ;
    HASE_CUDA(w.ensure(size_t(rows) * n));
    HASE_CUDA(dq.ensure(size_t(rows) * n));
    HASE_CUDA(doff.ensure(size_t(rows) * (n + 1)));
    HASE_CUDA(dph.ensure(rows));
    HASE_CUDA(dQ.ensure(rows));
    HASE_CUDA(cudaMemcpy(w.p, weights, size_t(rows) * n * sizeof(float), cudaMemcpyHostToDevice));
    HASE_CUDA(cudaMemcpy(dph.p, phases, rows * sizeof(uint32_t), cudaMemcpyHostToDevice));
    MapLaunch ml{w.p, 0, 1, nullptr, n, rays, dph.p, 0u, 0u, 0u, 0u, nullptr, dq.p, dQ.p, doff.p};
    mapKernel<<<rows, kMapBlock>>>(ml);
    HASE_CUDA(cudaGetLastError());
    HASE_CUDA(cudaDeviceSynchronize());
    HASE_CUDA(cudaMemcpy(q, dq.p, size_t(rows) * n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    HASE_CUDA(cudaMemcpy(offsets, doff.p, size_t(rows) * (n + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    std::vector<unsigned long long> hQ(rows);
    HASE_CUDA(cudaMemcpy(hQ.data(), dQ.p, rows * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < rows; ++i) Qout[i] = hQ[i];
    return HASE_OK;
}

hase_status hase_mesh_tables(const hase_mesh_desc* d, float* tri, float* walk) {
    if (!d || !d->points || !d->triangles || d->numberOfTriangles == 0)
        return fail(HASE_INVALID_ARGUMENT, "mesh points and triangles are required");
    HostTables ht;
    double extent = 0.0;
    const hase_status st = buildHostTables(d, ht, extent);
    if (st != HASE_OK) return st;
    const size_t bytes = ht.tri.size() * sizeof(float4);
    if (tri) std::memcpy(tri, ht.tri.data(), bytes);
    if (walk) std::memcpy(walk, ht.walk.data(), bytes);
    return HASE_OK;
}

hase_status hase_trace_rays(hase_context* c, uint32_t n, const float* start, const uint32_t* tri,
                            const uint32_t* level, const uint32_t* sample, const uint32_t* slice, uint32_t wavelength,
                            float* lnGain, float* distance, uint32_t* dropped) {
    if (!c || !start || !tri || !level || !sample || !slice || !lnGain || !distance || !dropped)
        return fail(HASE_INVALID_ARGUMENT, "null argument");
    if (n == 0) return HASE_OK;
    if (wavelength >= c->sigmaA.size()) return fail(HASE_INVALID_ARGUMENT, "wavelength index out of range");
    for (uint32_t i = 0; i < n; ++i) {
        if (tri[i] >= c->T || level[i] >= c->layers || sample[i] >= c->Np * c->L || slice[i] > 4)
            return fail(HASE_INVALID_ARGUMENT, "ray %u: index out of range", i);
    }
    HASE_TRY(setDevice(c));
    DevBuf<float> dStart, dLn, dDist;
    DevBuf<uint32_t> dTri, dLev, dSam, dSli, dDrop;
    HASE_CUDA(dStart.ensure(3 * size_t(n)));
    HASE_CUDA(dLn.ensure(n));
    HASE_CUDA(dDist.ensure(n));
    HASE_CUDA(dTri.ensure(n));
    HASE_CUDA(dLev.ensure(n));
    HASE_CUDA(dSam.ensure(n));
    HASE_CUDA(dSli.ensure(n));
    HASE_CUDA(dDrop.ensure(n));
    HASE_CUDA(cudaMemcpyAsync(dStart.p, start, 3 * size_t(n) * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    HASE_CUDA(cudaMemcpyAsync(dTri.p, tri, n * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
    HASE_CUDA(cudaMemcpyAsync(dLev.p, level, n * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
    HASE_CUDA(cudaMemcpyAsync(dSam.p, sample, n * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
    HASE_CUDA(cudaMemcpyAsync(dSli.p, slice, n * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
    const float A = float(c->nTot * (c->sigmaE[wavelength] + c->sigmaA[wavelength]));
    const float B = float(c->nTot * c->sigmaA[wavelength]);
    TraceLaunch tl{c->view(), n, dStart.p, dTri.p, dLev.p, dSam.p, dSli.p, A, B, dLn.p, dDist.p, dDrop.p};
    traceKernel<<<(n + 127) / 128, 128, 0, c->stream>>>(tl);
    HASE_CUDA(cudaGetLastError());
    HASE_CUDA(cudaMemcpyAsync(lnGain, dLn.p, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    HASE_CUDA(cudaMemcpyAsync(distance, dDist.p, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    HASE_CUDA(cudaMemcpyAsync(dropped, dDrop.p, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    HASE_CUDA(cudaStreamSynchronize(c->stream));
    return HASE_OK;
}

hase_status hase_philox(uint32_t n, const uint32_t* ctr, const uint32_t key[2], uint32_t* out) {
    if (!ctr || !key || !out) return fail(HASE_INVALID_ARGUMENT, "null argument");
    if (n == 0) return HASE_OK;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(HASE_NO_DEVICE, "no CUDA device available");
    }
    DevBuf<uint32_t> dc, dout;
    HASE_CUDA(dc.ensure(4 * size_t(n)));
    HASE_CUDA(dout.ensure(4 * size_t(n)));
    HASE_CUDA(cudaMemcpy(dc.p, ctr, 4 * size_t(n) * sizeof(uint32_t), cudaMemcpyHostToDevice));
    philoxKernel<<<(n + 127) / 128, 128>>>(n, dc.p, key[0], key[1], dout.p);
    HASE_CUDA(cudaGetLastError());
    HASE_CUDA(cudaDeviceSynchronize());
    HASE_CUDA(cudaMemcpy(out, dout.p, 4 * size_t(n) * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return HASE_OK;
}

hase_status hase_probe_l2_bandwidth(int device, uint64_t bytes, uint32_t reps, double* gbPerSecond) {
    if (!gbPerSecond || bytes < 1024 || reps == 0) return fail(HASE_INVALID_ARGUMENT, "bad argument");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(HASE_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= count) return fail(HASE_INVALID_ARGUMENT, "device out of range");
    HASE_CUDA(cudaSetDevice(device));
    const size_t n = size_t(bytes / 16);
    DevBuf<float4> buf;
    DevBuf<float> sink;
    HASE_CUDA(buf.ensure(n));
    HASE_CUDA(sink.ensure(1));
    HASE_CUDA(cudaMemset(buf.p, 0, n * sizeof(float4)));
    int sms = 0;
    HASE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    cudaEvent_t e0, e1;
    HASE_CUDA(cudaEventCreate(&e0));
    HASE_CUDA(cudaEventCreate(&e1));
    l2ProbeKernel<<<sms * 4, 512>>>(buf.p, n, 1, sink.p);  // warm the L2
    HASE_CUDA(cudaEventRecord(e0));
    l2ProbeKernel<<<sms * 4, 512>>>(buf.p, n, reps, sink.p);
    HASE_CUDA(cudaEventRecord(e1));
    HASE_CUDA(cudaGetLastError());
    HASE_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    HASE_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *gbPerSecond = double(n) * 16.0 * reps / (double(ms) * 1e-3) / 1e9;
    return HASE_OK;
}

hase_status hase_probe_l1_bandwidth(int device, uint32_t sharedMemory, uint32_t reps, double* gbPerSecond) {
    if (!gbPerSecond || reps == 0) return fail(HASE_INVALID_ARGUMENT, "bad argument");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(HASE_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= count) return fail(HASE_INVALID_ARGUMENT, "device out of range");
    HASE_CUDA(cudaSetDevice(device));
    DevBuf<float4> buf;
    DevBuf<float> sink;
    HASE_CUDA(buf.ensure(kProbeVec));
    HASE_CUDA(sink.ensure(1));
    HASE_CUDA(cudaMemset(buf.p, 0, kProbeVec * sizeof(float4)));
    int sms = 0;
    HASE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const uint32_t blocks = uint32_t(sms) * 2;  // two 1024-thread blocks per SM
    cudaEvent_t e0, e1;
    HASE_CUDA(cudaEventCreate(&e0));
    HASE_CUDA(cudaEventCreate(&e1));
    for (int pass = 0; pass < 2; ++pass) {  // the first pass warms the caches and the clocks
        const uint32_t r = pass == 0 ? 1u : reps;
        HASE_CUDA(cudaEventRecord(e0));
        if (sharedMemory) smemProbeKernel<<<blocks, 1024>>>(r, sink.p);
        else l1ProbeKernel<<<blocks, 1024>>>(buf.p, r, sink.p);
        HASE_CUDA(cudaEventRecord(e1));
        HASE_CUDA(cudaGetLastError());
    }
    HASE_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    HASE_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *gbPerSecond = double(blocks) * kProbeVec * 16.0 * reps / (double(ms) * 1e-3) / 1e9;
    return HASE_OK;
}

// hase_estimate_sample_noalloc: device address of g_noAllocScratch, looked up
// once per device (with that device current) on the first call there.
namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noAllocMutex;
unsigned char* g_noAllocPtr[kMaxDevices] = {};
}  // namespace

hase_status hase_estimate_sample_noalloc(hase_context* c, uint32_t sample, const float* deviceWeights, uint32_t rays,
                                         uint32_t rngSeed, uint32_t useReflections, uint32_t nearFieldSampling,
                                         double* deviceResult) {
    if (!c || !deviceWeights || !deviceResult) return fail(HASE_INVALID_ARGUMENT, "null argument");
    if (sample >= c->Np * c->L) return fail(HASE_INVALID_ARGUMENT, "sample %u out of range", sample);
    if (rays == 0 || rays > (1u << 31)) return fail(HASE_INVALID_ARGUMENT, "rays must be in [1, 2^31]");
    const uint32_t slices = useReflections ? 5u : 1u;
    const uint64_t nW = uint64_t(slices) * c->P;
    if (nW > kNoAllocMaxPrismSlices)
        return fail(HASE_INVALID_ARGUMENT,
                    "%llu prism slices exceed the allocation-free limit of %u (reflection slices x prisms)",
                    (unsigned long long)nW, kNoAllocMaxPrismSlices);
    if (c->device < 0 || c->device >= kMaxDevices) return fail(HASE_INVALID_ARGUMENT, "device index too large");
    HASE_TRY(setDevice(c));
    unsigned char* base;
    {
        std::lock_guard<std::mutex> lock(g_noAllocMutex);
        if (!g_noAllocPtr[c->device]) {
            void* ptr = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noAllocScratch);
            if (e != cudaSuccess || !ptr)
                return fail(HASE_CUDA_ERROR, "cudaGetSymbolAddress(g_noAllocScratch): %s", cudaGetErrorString(e));
            g_noAllocPtr[c->device] = static_cast<unsigned char*>(ptr);
        }
        base = g_noAllocPtr[c->device];
    }
    uint32_t* q = reinterpret_cast<uint32_t*>(base + kNoAllocQ);
    uint32_t* offsets = reinterpret_cast<uint32_t*>(base + kNoAllocOffsets);
    unsigned char* small = base + kNoAllocSmall;
    unsigned long long* Q = reinterpret_cast<unsigned long long*>(small + 0);
    uint32_t* active = reinterpret_cast<uint32_t*>(small + 8);
    unsigned int* itemCounter = reinterpret_cast<unsigned int*>(small + 12);
    uint32_t* nextActive = reinterpret_cast<uint32_t*>(small + 16);
    uint32_t* nextCount = reinterpret_cast<uint32_t*>(small + 20);
    double* accSum = reinterpret_cast<double*>(small + 24);
    double* accSum2 = reinterpret_cast<double*>(small + 32);
    uint32_t* accTotal = reinterpret_cast<uint32_t*>(small + 40);
    uint32_t* accDrop = reinterpret_cast<uint32_t*>(small + 44);
    unsigned long long* accCross = reinterpret_cast<unsigned long long*>(small + 48);
    float* phi = reinterpret_cast<float*>(small + 56);
    double* mse = reinterpret_cast<double*>(small + 64);
    unsigned char* parts = base + kNoAllocPartials;
    double* pSum = reinterpret_cast<double*>(parts);
    double* pSum2 = reinterpret_cast<double*>(parts + 8ull * kMaxItems);
    uint32_t* pDrop = reinterpret_cast<uint32_t*>(parts + 16ull * kMaxItems);
    unsigned long long* pCross = reinterpret_cast<unsigned long long*>(parts + 20ull * kMaxItems);

    // The scratch keeps the previous call's contents: clear what must start at zero.
    HASE_CUDA(cudaMemsetAsync(small, 0, 256, c->stream));  // Q, active = {row 0}, counters, accumulators
    const MeshView mv = c->view();
    MapLaunch ml{deviceWeights, 0, 1, active, uint32_t(nW), rays, nullptr, sample, 0u, rngSeed, 0u,
                 nullptr, q, Q, offsets};
    mapKernel<<<1, kMapBlock, 0, c->stream>>>(ml);
    HASE_CUDA(cudaGetLastError());
    const uint32_t itemRays = std::max<uint32_t>(kMinItemRays, (rays + kMaxItems - 1) / kMaxItems);
    const uint32_t items = (rays + itemRays - 1) / itemRays;
    const double C = c->nTot / (4.0 * kPi * c->tau);
    RayLaunch rl{mv, active, 1u, sample, 0u, rays, uint32_t(nW), itemRays, items, itemCounter, q, Q, offsets,
                 rngSeed, 0u, c->spec.p, uint32_t(c->sigmaA.size()), nearFieldSampling, C, pSum, pSum2, pDrop,
                 pCross};
    // row 0 addresses sample `sample`: the kernels index rows relative to firstSample
    const uint32_t grid = std::min<uint32_t>(items / (kRayBlock / 32) + 1, c->persistentBlocks);
    rayKernel<kRayBlock, kRefill, kRayMinBlocks><<<grid, kRayBlock, 0, c->stream>>>(rl);
    HASE_CUDA(cudaGetLastError());
    FinalizeLaunch fl{active, 1u, items, rays, 1, 0.0, pSum, pSum2, pDrop, pCross, accSum, accSum2, accTotal,
                      accDrop, accCross, phi, mse, nextActive, nextCount};
    finalizeKernel<<<1, 128, 0, c->stream>>>(fl);
    HASE_CUDA(cudaGetLastError());
    noAllocEmitKernel<<<1, 1, 0, c->stream>>>(phi, mse, accTotal, accDrop, deviceResult);
    HASE_CUDA(cudaGetLastError());
    HASE_CUDA(cudaStreamSynchronize(c->stream));
    return HASE_OK;
}

}  // extern "C"

// ------------------------------------------------- batched gain media ----
// hase_calc_phi_ase_batch: the sample points of many contexts in one pooled
// workspace, every adaptive pass one map, one persistent ray and one finalise
// launch over the active rows of all media, the whole schedule of a
// workspace chunk captured as one CUDA graph.

struct hase_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<cudaEvent_t> ev;  // timing events recorded inside the graphs
    DevBuf<float> lnw, phi, prior;
    DevBuf<uint8_t> rowFlag;      // rows restarting with the importance weights (learned solve)
    DevBuf<uint32_t> q, offsets, activeA, activeB, accTotal, accDrop, pDrop;
    DevBuf<unsigned int> counts;  // [0], [1]: active rows (alternating), [2]: item counter, [3 ..]: per pass
    DevBuf<unsigned long long> Q, accCross, pCross;
    DevBuf<double> accSum, accSum2, pSum, pSum2, mse;
    DevBuf<float2> spec;
    DevBuf<InstanceView> inst;
    DevBuf<RowInfo> rows;
    uint32_t variantBlocks[2][16] = {};  // general and no-cladding walks x launch shapes
    int sms = 0;
};

namespace {

struct BatchMedium {
    hase_context* c;
    uint32_t first, nS, nW, nLambda;
    double meanA, meanB, sA, sE;  // sA/sE: the pair of the dndt output
};

// Ends a stream capture that an error interrupted, so the stream stays usable.
struct CaptureGuard {
    cudaStream_t s;
    bool active = false;
    ~CaptureGuard() {
        if (active) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(s, &g);
            if (g) cudaGraphDestroy(g);
        }
    }
};

struct GraphOwner {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t x = nullptr;
    ~GraphOwner() {
        if (x) cudaGraphExecDestroy(x);
        if (g) cudaGraphDestroy(g);
    }
};

}  // namespace

extern "C" {

hase_status hase_batch_create(int device, hase_batch** out) {
    if (!out) return fail(HASE_INVALID_ARGUMENT, "null output pointer");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return fail(HASE_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= n) return fail(HASE_INVALID_ARGUMENT, "device %d outside [0, %d)", device, n);
    HASE_CUDA(cudaSetDevice(device));
    hase_batch* b = new (std::nothrow) hase_batch;
    if (!b) return fail(HASE_OUT_OF_MEMORY, "host allocation failed");
    b->device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) {
        delete b;
        return fail(HASE_CUDA_ERROR, "batch stream: %s", cudaGetErrorString(e));
    }
    *out = b;
    return HASE_OK;
}

hase_status hase_batch_destroy(hase_batch* b) {
    if (!b) return HASE_OK;
    cudaSetDevice(b->device);
    for (cudaEvent_t e : b->ev) cudaEventDestroy(e);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return HASE_OK;
}

}  // extern "C"

namespace {

// Checks the instances and fills the per-medium table (spectrum, sizes).
hase_status batchMedia(const hase_batch* b, const hase_batch_instance* in, uint32_t count,
                       const hase_experiment_desc* ex, std::vector<BatchMedium>& media,
                       std::vector<float2>& specPool, std::vector<uint32_t>& specBase) {
    const uint32_t slices = ex->useReflections ? 5u : 1u;
    media.resize(count);
    specPool.clear();
    specBase.resize(count);
    for (uint32_t i = 0; i < count; ++i) {
        hase_context* c = in[i].context;
        if (!c) return fail(HASE_INVALID_ARGUMENT, "instance %u has no context", i);
        if (c->device != b->device)
            return fail(HASE_INVALID_ARGUMENT, "instance %u is on device %d, the batch on %d", i, c->device, b->device);
        if (!in[i].result) return fail(HASE_INVALID_ARGUMENT, "instance %u has no result", i);
        if (c->localK) return fail(HASE_INVALID_ARGUMENT, "instance %u uses the local proposal, which batches do not", i);
        const uint32_t nTot = c->Np * c->L;
        const uint32_t first = in[i].minSample;
        const uint32_t last = in[i].maxSample == UINT32_MAX ? nTot - 1 : in[i].maxSample;
        if (first > last || last >= nTot)
            return fail(HASE_INVALID_ARGUMENT, "instance %u: sample range [%u, %u] outside [0, %u)", i, first, last,
                        nTot);
        if (uint64_t(slices) * c->P > 0xffffffffull)
            return fail(HASE_INVALID_ARGUMENT, "instance %u: too many prisms", i);
        BatchMedium& m = media[i];
        m.c = c;
        m.first = first;
        m.nS = last - first + 1;
        m.nW = slices * c->P;
        m.nLambda = ex->monochromatic ? 1u : uint32_t(c->sigmaA.size());
        m.meanA = m.meanB = m.sA = m.sE = 0.0;
        specBase[i] = uint32_t(specPool.size());
        for (uint32_t l = 0; l < m.nLambda; ++l) {
            const double A = c->nTot * (c->sigmaE[l] + c->sigmaA[l]), B = c->nTot * c->sigmaA[l];
            specPool.push_back(make_float2(float(A), float(B)));
            m.meanA += A / m.nLambda;
            m.meanB += B / m.nLambda;
            m.sA = std::max(m.sA, c->sigmaA[l]);
            m.sE = std::max(m.sE, c->sigmaE[l]);
        }
        if (m.nLambda == 1) {
            m.sA = c->sigmaA[0];
            m.sE = c->sigmaE[0];
        }
    }
    return HASE_OK;
}

}  // namespace

namespace {

// The batched solve; net != null: every medium's importance weights are
// replaced by the learned proposal (network logits mixed with the
// beta V R_j / d^2 prior, weight alpha), as hase_calc_phi_ase_learned does.
hase_status batchCore(hase_batch* b, const hase_batch_instance* in, uint32_t count, const hase_experiment_desc* ex,
                      const hase_compute_desc* cp, hase_batch_stats* stats, hase_proposal* net, float alpha,
                      float fallbackVariance) {
    if (!b || !in || !ex || !cp || count == 0) return fail(HASE_INVALID_ARGUMENT, "null argument or no instances");
    const auto hostStart = std::chrono::steady_clock::now();
    auto sinceStart = [&] {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - hostStart).count();
    };
    if (ex->minRays == 0) return fail(HASE_INVALID_ARGUMENT, "minRays must be positive");
    if (ex->maxRays != 0 && ex->maxRays < ex->minRays) return fail(HASE_INVALID_ARGUMENT, "maxRays < minRays");
    if (!(ex->mseThreshold >= 0.0)) return fail(HASE_INVALID_ARGUMENT, "mseThreshold must be >= 0");
    if (!validImportanceLayers(cp->importanceLayers))
        return fail(HASE_INVALID_ARGUMENT, "importanceLayers must be 0, 2, 4 or 8");
    if (cp->rayKernelVariant >= kNumRayVariants)
        return fail(HASE_INVALID_ARGUMENT, "rayKernelVariant %u >= %u", cp->rayKernelVariant, kNumRayVariants);
    HASE_CUDA(cudaSetDevice(b->device));
    std::vector<BatchMedium> media;
    std::vector<float2> specPool;
    std::vector<uint32_t> specBase;
    HASE_TRY(batchMedia(b, in, count, ex, media, specPool, specBase));
    const uint32_t maxRays = std::max(ex->maxRays, ex->minRays);
    const uint32_t slices = ex->useReflections ? 5u : 1u;
    const uint32_t variant = cp->rayKernelVariant;
    const RayVariant& rv = kPoolVariants[variant];
    if (b->variantBlocks[0][variant] == 0) {
        for (int w = 0; w < 2; ++w) {
            int perSM = 0;
            HASE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, w ? rv.noClad : rv.kernel, rv.block, 0));
            b->variantBlocks[w][variant] = uint32_t(std::max(1, perSM) * std::max(1, b->sms));
        }
    }
    // a batch without cladding prisms walks without the per-crossing cladding test
    bool anyClad = false;
    for (const BatchMedium& md : media) anyClad = anyClad || md.c->hasClad;
    const int noClad = anyClad ? 0 : 1;

    // the pass schedule (shared by all media)
    struct Pass {
        uint32_t M, itemRays, items;
        bool last;
    };
    std::vector<Pass> passes;
    for (uint32_t pass = 0, prev = 0;; ++pass) {
        const uint32_t target = adaptiveTarget(ex->minRays, maxRays, cp->adaptiveSteps, pass);
        const bool last = target >= maxRays || pass >= cp->adaptiveSteps;
        Pass ps;
        ps.M = target - prev;
        ps.itemRays = std::max<uint32_t>(cp->raysPerThread ? 32u * cp->raysPerThread : kMinItemRays,
                                         (ps.M + kMaxItems - 1) / kMaxItems);
        ps.items = (ps.M + ps.itemRays - 1) / ps.itemRays;
        ps.last = last;
        passes.push_back(ps);
        prev = target;
        if (last) break;
    }
    const uint32_t nPasses = uint32_t(passes.size());

    // media views and spectra
    HASE_CUDA(b->spec.ensure(specPool.size()));
    HASE_CUDA(b->inst.ensure(count));
    std::vector<InstanceView> views(count);
    for (uint32_t i = 0; i < count; ++i) {
        const hase_context* c = media[i].c;
        InstanceView& v = views[i];
        std::memset(&v, 0, sizeof(v));
        v.m = c->view();
        v.spec = b->spec.p + specBase[i];
        v.nLambda = media[i].nLambda;
        v.nW = media[i].nW;
        v.seedLo = cp->rngSeed + i;
        v.C = c->nTot / (4.0 * kPi * c->tau);
    }
    HASE_CUDA(cudaMemcpyAsync(b->spec.p, specPool.data(), specPool.size() * sizeof(float2), cudaMemcpyHostToDevice,
                              b->stream));
    HASE_CUDA(cudaMemcpyAsync(b->inst.p, views.data(), count * sizeof(InstanceView), cudaMemcpyHostToDevice,
                              b->stream));
    // learned proposal: one feature view per medium (coarse gain grid on the medium's context)
    std::vector<ProposalView> pviews;
    uint32_t proposalGrid = 0;
    if (net) {
        if (net->device != b->device)
            return fail(HASE_INVALID_ARGUMENT, "the proposal network and the batch are on different devices");
        pviews.resize(count);
        for (uint32_t i = 0; i < count; ++i) {
            HASE_TRY(cachedProposalView(media[i].c, media[i].meanA, media[i].meanB, pviews[i]));
            pviews[i].nW = media[i].nW;
        }
        HASE_CUDA(cudaFuncSetAttribute(proposalKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemBytes)));
        proposalGrid = uint32_t(std::max(1, b->sms) * kMlpBlocksPerSM);
    } else {
        // media whose context takes the coarse-grid proposal: their views
        pviews.resize(count);
        for (uint32_t i = 0; i < count; ++i)
            if (media[i].c->gridProposal) {
                HASE_TRY(cachedProposalView(media[i].c, media[i].meanA, media[i].meanB, pviews[i]));
                pviews[i].nW = media[i].nW;
            }
    }
    // the views' gain grids are built on each context's own stream: finished
    // before the batch's stream reads them
    for (uint32_t i = 0; i < count; ++i) HASE_CUDA(cudaStreamSynchronize(media[i].c->stream));

    // rows of every medium, cut into workspace chunks
    struct Chunk {
        size_t r0, r1;            // global rows [r0, r1)
        unsigned long long ws;    // workspace entries (sum of nW)
    };
    std::vector<RowInfo> all;
    for (uint32_t i = 0; i < count; ++i) {
        all.reserve(all.size() + media[i].nS);
        for (uint32_t s = 0; s < media[i].nS; ++s) all.push_back(RowInfo{0ull, i, media[i].first + s, media[i].nW,
                                                                           cp->rngSeed + i});
    }
    const uint64_t budget = cp->workspaceBytes ? cp->workspaceBytes : (uint64_t(4) << 30);
    std::vector<Chunk> chunks;
    {
        Chunk ch{0, 0, 0};
        uint64_t bytes = 0;
        for (size_t r = 0; r < all.size(); ++r) {
            const uint64_t perRow = uint64_t(all[r].nW) * 12 + 16 + kMaxItems * 28ull + 64;
            if (ch.r1 > ch.r0 && bytes + perRow > budget) {
                chunks.push_back(ch);
                ch = Chunk{r, r, 0};
                bytes = 0;
            }
            all[r].w = ch.ws;
            ch.ws += all[r].nW;
            ch.r1 = r + 1;
            bytes += perRow;
        }
        chunks.push_back(ch);
    }
    size_t maxRows = 0;
    unsigned long long maxWs = 0;
    for (const Chunk& ch : chunks) {
        maxRows = std::max(maxRows, ch.r1 - ch.r0);
        maxWs = std::max(maxWs, ch.ws);
    }
    if (maxRows > 0xffffffffull) return fail(HASE_INVALID_ARGUMENT, "too many sample points in one chunk");
    HASE_CUDA(b->lnw.ensure(maxWs));
    if (net) HASE_CUDA(b->prior.ensure(maxWs));
    HASE_CUDA(b->q.ensure(maxWs));
    HASE_CUDA(b->offsets.ensure(maxWs + maxRows));
    HASE_CUDA(b->Q.ensure(maxRows));
    HASE_CUDA(b->rows.ensure(maxRows));
    HASE_CUDA(b->activeA.ensure(maxRows));
    HASE_CUDA(b->activeB.ensure(maxRows));
    HASE_CUDA(b->counts.ensure(4 + nPasses));
    const bool fallback = net && fallbackVariance > 0.0f && nPasses > 1;
    if (fallback) HASE_CUDA(b->rowFlag.ensure(maxRows));
    HASE_CUDA(b->accSum.ensure(maxRows));
    HASE_CUDA(b->accSum2.ensure(maxRows));
    HASE_CUDA(b->accTotal.ensure(maxRows));
    HASE_CUDA(b->accDrop.ensure(maxRows));
    HASE_CUDA(b->accCross.ensure(maxRows));
    HASE_CUDA(b->phi.ensure(maxRows));
    HASE_CUDA(b->mse.ensure(maxRows));
    HASE_CUDA(b->pSum.ensure(maxRows * kMaxItems));
    HASE_CUDA(b->pSum2.ensure(maxRows * kMaxItems));
    HASE_CUDA(b->pDrop.ensure(maxRows * kMaxItems));
    HASE_CUDA(b->pCross.ensure(maxRows * kMaxItems));
    const size_t nEvents = 3 + 2 * size_t(nPasses);
    while (b->ev.size() < nEvents) {
        cudaEvent_t e = nullptr;
        HASE_CUDA(cudaEventCreate(&e));
        b->ev.push_back(e);
    }

    hase_batch_stats st{};
    st.rows = uint32_t(all.size());
    st.chunks = uint32_t(chunks.size());
    std::vector<uint32_t> unconvergedOf(count, 0), passesOf(count, 0);
    std::vector<uint64_t> raysOf(count, 0), crossOf(count, 0);
    uint64_t droppedTotal = 0;
    std::vector<float> hPhi(maxRows);
    std::vector<double> hMse(maxRows);
    std::vector<uint32_t> hTotal(maxRows), hDrop(maxRows), hCounts(4 + nPasses);
    std::vector<unsigned long long> hCross(maxRows);
    const double thr = ex->mseThreshold;

    for (const Chunk& ch : chunks) {
        const uint32_t nRows = uint32_t(ch.r1 - ch.r0);
        if (&ch == &chunks.front()) st.setupMilliseconds = sinceStart();
        HASE_CUDA(cudaMemcpyAsync(b->rows.p, all.data() + ch.r0, nRows * sizeof(RowInfo), cudaMemcpyHostToDevice,
                                  b->stream));
        HASE_CUDA(cudaStreamSynchronize(b->stream));
        const auto tc0 = std::chrono::steady_clock::now();
        GraphOwner graph;
        uint32_t kernels = 0;
        {
            CaptureGuard guard{b->stream};
            HASE_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            guard.active = true;
            HASE_CUDA(cudaEventRecordWithFlags(b->ev[0], b->stream, cudaEventRecordExternal));
            // importance weights of the rows [r, e) of one medium (only the flagged ones with a flag array)
            auto importanceSegment = [&](size_t r, size_t e, const uint8_t* flag) -> hase_status {
                const uint32_t i = all[r].inst;
                const BatchMedium& md = media[i];
                const hase_context* c = md.c;
                const uint32_t segRows = uint32_t(e - r);
                ImportanceLaunch il{views[i].m, all[r].sample, slices, md.nW, float(md.meanA), float(md.meanB),
                                    b->lnw.p + all[r].w, nullptr, flag, uint32_t(r - ch.r0)};
                HASE_CUDA(launchImportance(cp->importanceLayers, il, c->layers, c->T, segRows, b->stream));
                ++kernels;
                return HASE_OK;
            };
            // runs of rows of one medium (at most 65,535 rows each: the grid's y extent)
            std::vector<std::pair<size_t, size_t>> segments;
            for (size_t r = ch.r0; r < ch.r1;) {
                size_t e = r;
                while (e < ch.r1 && all[e].inst == all[r].inst && e - r < 65535) ++e;
                segments.emplace_back(r, e);
                r = e;
            }
            // (a1) importance weights or the learned proposal, one launch per run of rows of one medium
            for (const auto& seg : segments) {
                const size_t r = seg.first, e = seg.second;
                const uint32_t i = all[r].inst;
                const BatchMedium& md = media[i];
                const uint32_t segRows = uint32_t(e - r);
                if (net) {
                    ProposalView pv = pviews[i];
                    pv.firstSample = all[r].sample;
                    ProposalLaunch pl{pv, net->wimg.p, net->vec.p, b->lnw.p + all[r].w, b->prior.p + all[r].w,
                                      nullptr, segRows, net->error.p};
                    const uint64_t tiles = (uint64_t(segRows) * md.nW + kTile - 1) / kTile;
                    proposalKernel<<<uint32_t(std::min<uint64_t>(tiles, proposalGrid)), kTile, kSmemBytes,
                                     b->stream>>>(pl);
                    HASE_CUDA(cudaGetLastError());
                    mixtureKernel<<<segRows, 1024, 0, b->stream>>>(md.nW, b->lnw.p + all[r].w, b->prior.p + all[r].w,
                                                                  alpha);
                    kernels += 2;
                } else if (md.c->gridProposal) {
                    ProposalView pv = pviews[i];
                    pv.firstSample = all[r].sample;
                    const ProposalLaunch gl{pv, nullptr, nullptr, b->lnw.p + all[r].w, nullptr, nullptr, segRows,
                                            nullptr};
                    HASE_CUDA(launchGridWeights(gl, b->stream));
                    ++kernels;
                } else {
                    HASE_TRY(importanceSegment(r, e, nullptr));
                }
                HASE_CUDA(cudaGetLastError());
            }
            HASE_CUDA(cudaEventRecordWithFlags(b->ev[1], b->stream, cudaEventRecordExternal));
            HASE_CUDA(cudaMemsetAsync(b->accSum.p, 0, nRows * sizeof(double), b->stream));
            HASE_CUDA(cudaMemsetAsync(b->accSum2.p, 0, nRows * sizeof(double), b->stream));
            HASE_CUDA(cudaMemsetAsync(b->accTotal.p, 0, nRows * sizeof(uint32_t), b->stream));
            HASE_CUDA(cudaMemsetAsync(b->accDrop.p, 0, nRows * sizeof(uint32_t), b->stream));
            HASE_CUDA(cudaMemsetAsync(b->accCross.p, 0, nRows * sizeof(unsigned long long), b->stream));
            HASE_CUDA(cudaMemsetAsync(b->counts.p, 0, (4 + nPasses) * sizeof(unsigned int), b->stream));
            iotaCountKernel<<<(nRows + 255) / 256, 256, 0, b->stream>>>(b->activeA.p, nRows, b->counts.p);
            HASE_CUDA(cudaGetLastError());
            ++kernels;
            uint32_t* cur = b->activeA.p;
            uint32_t* nxt = b->activeB.p;
            unsigned int* cntCur = b->counts.p;
            unsigned int* cntNxt = b->counts.p + 1;
            unsigned int* itemCounter = b->counts.p + 2;
            const uint32_t mapGrid = std::min<uint32_t>(nRows, uint32_t(2 * b->sms));
            const uint32_t finGrid = std::min<uint32_t>((nRows * 32u + 127u) / 128u, uint32_t(16 * b->sms));
            for (uint32_t k = 0; k < nPasses; ++k) {
                const Pass& ps = passes[k];
                HASE_CUDA(cudaMemcpyAsync(b->counts.p + 3 + k, cntCur, sizeof(unsigned int), cudaMemcpyDeviceToDevice,
                                          b->stream));
                MapLaunch ml{b->lnw.p, 1, k == 0 ? 1 : 0, cur, 0u, ps.M, nullptr, 0u, k, 0u, 0u, nullptr, b->q.p,
                             b->Q.p, b->offsets.p, b->rows.p, cntCur};
                mapKernel<<<mapGrid, kMapBlock, 0, b->stream>>>(ml);
                HASE_CUDA(cudaGetLastError());
                HASE_CUDA(cudaMemsetAsync(itemCounter, 0, sizeof(unsigned int), b->stream));
                HASE_CUDA(cudaEventRecordWithFlags(b->ev[3 + 2 * k], b->stream, cudaEventRecordExternal));
                RayLaunch rl{};
                rl.active = cur;
                rl.pass = k;
                rl.M = ps.M;
                rl.itemRays = ps.itemRays;
                rl.itemsPerRow = ps.items;
                rl.itemCounter = itemCounter;
                rl.q = b->q.p;
                rl.Q = b->Q.p;
                rl.offsets = b->offsets.p;
                rl.nearField = ex->nearFieldSampling;
                rl.pSum = b->pSum.p;
                rl.pSum2 = b->pSum2.p;
                rl.pDrop = b->pDrop.p;
                rl.pCross = b->pCross.p;
                rl.inst = b->inst.p;
                rl.rows = b->rows.p;
                rl.count = cntCur;
                const uint32_t grid = uint32_t(std::min<uint64_t>(uint64_t(nRows) * ps.items / (rv.block / 32) + 1,
                                                                   uint64_t(b->variantBlocks[noClad][variant])));
                void* rayArgs[] = {&rl};
                HASE_CUDA(cudaLaunchKernel(reinterpret_cast<const void*>(noClad ? rv.noClad : rv.kernel), dim3(grid),
                                           dim3(rv.block), rayArgs, 0, b->stream));
                HASE_CUDA(cudaEventRecordWithFlags(b->ev[4 + 2 * k], b->stream, cudaEventRecordExternal));
                HASE_CUDA(cudaMemsetAsync(cntNxt, 0, sizeof(unsigned int), b->stream));
                FinalizeLaunch fl{cur, 0u, ps.items, ps.M, ps.last ? 1 : 0, thr, b->pSum.p, b->pSum2.p, b->pDrop.p,
                                  b->pCross.p, b->accSum.p, b->accSum2.p, b->accTotal.p, b->accDrop.p, b->accCross.p,
                                  b->phi.p, b->mse.p, nxt, cntNxt, cntCur};
                finalizeKernel<<<finGrid, 128, 0, b->stream>>>(fl);
                HASE_CUDA(cudaGetLastError());
                kernels += 3;
                std::swap(cur, nxt);
                std::swap(cntCur, cntNxt);
                if (fallback && k == 0) {
                    // the plain method judges: rows still active after the first pass whose per-ray
                    // variance under the learned proposal exceeds the limit restart with the
                    // importance weights (as hase_calc_phi_ase_learned does, on the device)
                    const uint32_t g = std::min<uint32_t>((nRows + 255) / 256, uint32_t(8 * b->sms));
                    HASE_CUDA(cudaMemsetAsync(b->rowFlag.p, 0, nRows, b->stream));
                    fallbackMarkKernel<<<g, 256, 0, b->stream>>>(cur, cntCur, b->accTotal.p, b->mse.p,
                                                                 double(fallbackVariance), b->rowFlag.p,
                                                                 b->counts.p + 3 + nPasses);
                    HASE_CUDA(cudaGetLastError());
                    for (const auto& seg : segments) HASE_TRY(importanceSegment(seg.first, seg.second, b->rowFlag.p));
                    MapLaunch rq{b->lnw.p, 1, 1, cur, 0u, 1u, nullptr, 0u, 0u, 0u, 0u, nullptr, b->q.p, b->Q.p,
                                 b->offsets.p, b->rows.p, cntCur, b->rowFlag.p};
                    mapKernel<<<mapGrid, kMapBlock, 0, b->stream>>>(rq);
                    resetFlaggedKernel<<<g, 256, 0, b->stream>>>(cur, cntCur, b->rowFlag.p, b->accSum.p, b->accSum2.p,
                                                                 b->accTotal.p, b->accDrop.p, b->accCross.p);
                    HASE_CUDA(cudaGetLastError());
                    kernels += 3;
                }
            }
            // after the last pass cntCur holds the samples above the threshold at maxRays
            if (cntCur != b->counts.p)
                HASE_CUDA(cudaMemcpyAsync(b->counts.p, cntCur, sizeof(unsigned int), cudaMemcpyDeviceToDevice,
                                          b->stream));
            HASE_CUDA(cudaEventRecordWithFlags(b->ev[2], b->stream, cudaEventRecordExternal));
            guard.active = false;
            HASE_CUDA(cudaStreamEndCapture(b->stream, &graph.g));
        }
        HASE_CUDA(cudaGraphInstantiate(&graph.x, graph.g, 0));
        size_t nodes = 0;
        HASE_CUDA(cudaGraphGetNodes(graph.g, nullptr, &nodes));
        st.captureMilliseconds +=
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tc0).count();
        HASE_CUDA(cudaGraphLaunch(graph.x, b->stream));
        HASE_CUDA(cudaMemcpyAsync(hPhi.data(), b->phi.p, nRows * sizeof(float), cudaMemcpyDeviceToHost, b->stream));
        HASE_CUDA(cudaMemcpyAsync(hMse.data(), b->mse.p, nRows * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
        HASE_CUDA(cudaMemcpyAsync(hTotal.data(), b->accTotal.p, nRows * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                  b->stream));
        HASE_CUDA(cudaMemcpyAsync(hDrop.data(), b->accDrop.p, nRows * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                  b->stream));
        HASE_CUDA(cudaMemcpyAsync(hCross.data(), b->accCross.p, nRows * sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, b->stream));
        HASE_CUDA(cudaMemcpyAsync(hCounts.data(), b->counts.p, (4 + nPasses) * sizeof(unsigned int),
                                  cudaMemcpyDeviceToHost, b->stream));
        HASE_CUDA(cudaStreamSynchronize(b->stream));
        float ms = 0.0f;
        HASE_CUDA(cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]));
        st.importanceMilliseconds += ms;
        HASE_CUDA(cudaEventElapsedTime(&ms, b->ev[0], b->ev[2]));
        st.totalMilliseconds += ms;
        for (uint32_t k = 0; k < nPasses; ++k) {
            HASE_CUDA(cudaEventElapsedTime(&ms, b->ev[3 + 2 * k], b->ev[4 + 2 * k]));
            st.rayMilliseconds += ms;
            if (hCounts[3 + k] > 0) st.passes = std::max(st.passes, k + 1);
        }
        st.unconvergedSamples += hCounts[0];
        st.fallbackSamples += fallback ? hCounts[3 + nPasses] : 0u;
        st.kernelLaunches += kernels;
        st.graphNodes += uint32_t(nodes);
        // scatter the chunk's rows into the media's results
        for (uint32_t j = 0; j < nRows; ++j) {
            const RowInfo& ri = all[ch.r0 + j];
            const BatchMedium& md = media[ri.inst];
            hase_result* res = in[ri.inst].result;
            const uint32_t o = ri.sample - md.first;
            if (res->phiAse) res->phiAse[o] = hPhi[j];
            if (res->relativeStandardError) res->relativeStandardError[o] = hMse[j];
            if (res->standardError) res->standardError[o] = hMse[j] * double(hPhi[j]);
            if (res->totalRays) res->totalRays[o] = hTotal[j];
            if (res->droppedRays) res->droppedRays[o] = hDrop[j];
            if (res->dndtAse) {
                const double bc = md.c->betaCells.empty() ? 0.0 : md.c->betaCells[ri.sample];
                res->dndtAse[o] = (bc * (md.sE + md.sA) - md.sA) * double(hPhi[j]);
            }
            if (!(hMse[j] <= thr)) ++unconvergedOf[ri.inst];
            uint32_t np = 0;
            for (uint32_t k = 0, cum = 0; k < nPasses && cum < hTotal[j]; ++k) {
                cum += passes[k].M;
                np = k + 1;
            }
            passesOf[ri.inst] = std::max(passesOf[ri.inst], np);
            raysOf[ri.inst] += hTotal[j];
            crossOf[ri.inst] += hCross[j];
            droppedTotal += hDrop[j];
            st.raysTraced += hTotal[j];
            st.crossings += hCross[j];
        }
    }
    for (uint32_t i = 0; i < count; ++i) {
        hase_result* res = in[i].result;
        res->raysTraced = raysOf[i];
        res->crossings = crossOf[i];
        res->unconvergedSamples = unconvergedOf[i];
        res->passes = passesOf[i];
        res->importanceMilliseconds = st.importanceMilliseconds;
        res->rayMilliseconds = st.rayMilliseconds;
        res->totalMilliseconds = st.totalMilliseconds;
        res->kernelLaunches = st.kernelLaunches;
    }
    st.hostMilliseconds = sinceStart();
    if (stats) *stats = st;
    if (net) {
        int err = 0;
        HASE_CUDA(cudaMemcpy(&err, net->error.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (err) return fail(HASE_DEVICE_TIMEOUT, "a tensor-core wait of the proposal network timed out");
    }
    if (droppedTotal) {
        fail(HASE_DROPPED_RAYS, "%llu rays could not be walked", (unsigned long long)droppedTotal);
        return HASE_DROPPED_RAYS;
    }
    if (st.unconvergedSamples) {
        fail(HASE_NOT_CONVERGED, "%u samples above the threshold at maxRays", st.unconvergedSamples);
        return HASE_NOT_CONVERGED;
    }
    return HASE_OK;
}

}  // namespace

extern "C" {

hase_status hase_calc_phi_ase_batch(hase_batch* b, const hase_batch_instance* in, uint32_t count,
                                    const hase_experiment_desc* ex, const hase_compute_desc* cp,
                                    hase_batch_stats* stats) {
    return batchCore(b, in, count, ex, cp, stats, nullptr, 0.0f, 0.0f);
}

hase_status hase_calc_phi_ase_batch_learned(hase_batch* b, const hase_batch_instance* in, uint32_t count,
                                            const hase_experiment_desc* ex, const hase_compute_desc* cp,
                                            hase_proposal* net, float mixture, float fallbackVariance,
                                            hase_batch_stats* stats) {
    if (!net) return fail(HASE_INVALID_ARGUMENT, "null network");
    if (!(mixture >= 0.0f) || mixture >= 1.0f) return fail(HASE_INVALID_ARGUMENT, "mixture must be in [0, 1)");
    if (!(fallbackVariance >= 0.0f)) return fail(HASE_INVALID_ARGUMENT, "fallbackVariance must be >= 0");
    return batchCore(b, in, count, ex, cp, stats, net, mixture > 0.0f ? mixture : 0.1f, fallbackVariance);
}

}  // extern "C"
