// hase_forward.cu -- the forward Tet4 phi-ASE path of libhase_b200.so
// (HASEonGPU v2.2.0's current calcPhiASE), FP64 on sm_100a.
//
// Per adaptive launch of M source rays, split round-robin over B statistical
// batches (ray r -> batch r % B, index r / B inside it):
//   fwdRayKernel   each block serves one batch; each lane owns a sequence of
//                  rays and starts the next one as soon as its current ray has
//                  left the mesh, so a warp stays full until the tail.  Source:
//                  stratified beta*V CDF target (i + shift_b)/N_b * B_tot and a
//                  binary search of the inclusive prefix, a uniform point in
//                  the tet from four exponentials (paired with the corners in
//                  ascending point index), an isotropic direction, a
//                  wavelength bin from a golden-ratio sequence over the
//                  batch's rays.  Walk: per cell the four
//                  barycentric face coordinates lambda_f = a.x + d and their
//                  rates along the ray; the exit is the decreasing coordinate
//                  that reaches zero first (cross-multiplied comparisons, one
//                  division per crossing).  Tally: weight G (e^{gl} - 1)/g split
//                  to the cell's four material vertices by the segment-midpoint
//                  barycentric weights, into a per-block shared-memory vertex
//                  histogram of the block's batch (flushed once per block) or,
//                  for meshes whose histogram does not fit, straight into
//                  device memory.
//   fwdFinalizeKernel  one thread per cell: vertex -> cell density through
//                  the lumped material-vertex volumes, estimate
//                  S B_tot / (N V) N_tot / tau, batch-mean relative error,
//                  dndt, and the count of cells above the threshold.
// Reference anchors (paths inside the HASEonGPU tree):
//   include/kernels/forward/accumulation.hpp:300-453 (kernel, tally),
//   include/kernels/forward/volumeSampling.hpp:19-161 (source sampling),
//   include/kernels/forward/rayWalk.hpp:106-208 (exit face, segment gain),
//   include/kernels/forwardPhiAseMapping.hpp:51-150 and
//   include/kernels/vertexAccumulation.hpp:17-68 (finaliser),
//   include/core/forwardPhiAseEvaluator.hpp:114-178 (adaptive launches),
//   include/core/mesh.hpp:657-727 (barycentric face planes).
#include "hase_b200_forward.h"
#include "hase_device.cuh"
#include "hase_host.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <map>
#include <new>
#include <tuple>
#include <vector>

using namespace hase;

namespace {

constexpr uint32_t kTagFwdBatch = 2u;  // Philox counter tags of the forward streams
constexpr uint32_t kTagFwdRay = 3u;
constexpr uint32_t kFwdKeyHi = 1u;     // key = {seed, 1}
constexpr uint32_t kMaxBatches = 64u;
constexpr uint32_t kFwdBlock = 256u;
constexpr int kFwdRefill = 8;          // idle lanes that trigger a batched start of new rays
constexpr int kFwdMinBlocks = 3;       // resident ray-kernel blocks per SM the register budget is cut for
constexpr int kFwdMaxSteps = 10000;    // bounded walk: a ray still inside after this many cells is dropped
constexpr int kFwdSteps = 32;         // cells a lane walks between the warp's ray-claim checks
constexpr size_t kMaxHistogramBytes = 200u * 1024u;
constexpr double kTwoPi = 6.283185307179586476925286766559;

// One cell's walk record: one 128-byte line.  Corners are stored sorted by
// global point index (face k opposite corner k), so that when a ray crosses
// from one cell into its neighbour the three shared corners keep their
// relative order: the old corners other than the exit face map, in order, to
// the new corners other than the entry face.  Only the planes of faces 1..3
// are stored; lambda_0 = 1 - (lambda_1 + lambda_2 + lambda_3) and its rate
// along the ray is minus the sum of theirs.
struct __align__(128) TetCell {
    double4 plane[3];  // faces 1..3: lambda_f(x) = a.x + b.y + c.z + d
    int4 nbr;          // per face (neighbour << 2) | neighbour's local face, -1 at the boundary
    uint4 matv;        // material vertex of each corner (cladding cells offset by Np)
};
static_assert(sizeof(TetCell) == 128, "TetCell must be one 128-byte line");

struct TetView {
    const TetCell* cell;    // [C]
    const double* gainBeta; // [C]: beta, NaN for cladding cells
    const double* points;   // [Np][3]
    const double* prefix;   // [C]: inclusive prefix of beta * V
    const uint32_t* guide;  // [K + 1]: guide[j] = first cell whose prefix exceeds j Btot / K; guide[K] = C
    uint32_t C, Np, lastSource, K;
    double cladAbs, nTot, Btot, guideScale;  // guideScale = K / Btot
};

__device__ __forceinline__ double unit53(uint32_t x) { return (double(x >> 8) + 0.5) * (1.0 / 16777216.0); }

// 256-bit read-only loads (sm_100): one 32-byte sector per lane and instruction.
__device__ __forceinline__ double4 ldPlane(const double4* p) {
    double4 v;
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w) : "l"(p));
    return v;
}

struct CellLinks {
    int4 nbr;
    uint4 matv;
};

__device__ __forceinline__ CellLinks ldLinks(const int4* p) {
    CellLinks l;
    asm("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(l.nbr.x), "=r"(l.nbr.y), "=r"(l.nbr.z), "=r"(l.nbr.w), "=r"(l.matv.x), "=r"(l.matv.y),
          "=r"(l.matv.z), "=r"(l.matv.w)
        : "l"(p));
    return l;
}

// Exit face of the cell whose planes of faces 1..3 are pl for a ray at (x, y, z) moving
// along u, the entry face ff excluded: among the faces with dlambda < 0, the
// smallest max(lambda, 0) / -dlambda (lowest index on a tie).  Fills lam and
// dl for all four faces; returns -1 when no face decreases.
__device__ __forceinline__ int exitFace(const double4* __restrict__ pl, double x, double y, double z, double ux,
                                        double uy, double uz, int ff, double lam[4], double dl[4], double& len) {
    int bf = -1;
    double bl = 0.0, bd = -1.0;
#pragma unroll
    for (int f = 1; f < 4; ++f) {
        const double4 p = ldPlane(pl + f - 1);
        lam[f] = fma(p.x, x, fma(p.y, y, fma(p.z, z, p.w)));
        dl[f] = fma(p.x, ux, fma(p.y, uy, p.z * uz));
    }
    lam[0] = 1.0 - (lam[1] + lam[2] + lam[3]);
    dl[0] = -(dl[1] + dl[2] + dl[3]);
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        if (f == ff || !(dl[f] < 0.0)) continue;
        const double lc = fmax(lam[f], 0.0);
        // lc / -dl[f] < bl / -bd  <=>  lc * bd > bl * dl[f]   (both rates negative)
        if (bf < 0 || lc * bd > bl * dl[f]) {
            bf = f;
            bl = lc;
            bd = dl[f];
        }
    }
    len = bf < 0 ? 0.0 : -bl / bd;
    return bf;
}

__device__ __forceinline__ double gainCoefficient(const TetView& m, uint32_t c, double sA, double sE) {
    const double beta = __ldg(m.gainBeta + c);
    return isnan(beta) ? -m.cladAbs : m.nTot * (beta * (sE + sA) - sA);
}

struct FwdRay {
    double x, y, z, ux, uy, uz, G, sA, sE;
    double pv[4];  // tallies not yet added to device memory, per corner of the current cell
    uint4 pid;     // the current cell's material vertices (owners of pv)
    int4 nbr;      // the current cell's neighbours (-1: boundary, <= -2: reflecting boundary face -2 - n)
    uint32_t c;
    int ff, steps;
    uint32_t id, lam;  // ray index of the launch, wavelength bin (reflection deposits)
};

// ---- surface-reservoir reflections ----
// A boundary face with a reflecting surface: outward unit normal, centroid
// (start point of the reflected rays), reflectivity, squared index ratio
// n_in / n_out (-1: no total internal reflection), its cell and the cell
// record's (corner-sorted) local face.
struct __align__(16) BFace {
    double n[3], cen[3], R, ratio2;
    uint32_t c, f, pad[2];
};
static_assert(sizeof(BFace) == 80, "BFace layout");

// One batch's reflection chain (include/core/forwardSrm.hpp:281-363).
struct SrmChain {
    double initial, prev, remaining;
    uint32_t grow, status, passes, active;
};

enum : uint32_t { kSrmDisabled = 0, kSrmConverged = 1, kSrmStable = 2, kSrmDiverged = 3, kSrmMaxIterations = 4 };

struct SrmLaunch {
    const BFace* faces;  // [nF]
    uint32_t nF, S, pass;
    // reservoir the launch deposits into: [B][nF] counts and weights, [B][nF][S] slots
    uint32_t* outCounts;
    double* outFaceW;
    double4* outSlot;    // reflected direction, weight
    uint32_t* outLam;
    uint32_t* outRay;    // ray index of the deposit (slot order; see srmSortKernel)
    // reservoir the reflected rays are drawn from, and the inclusive CDF of its face weights per batch
    const uint32_t* inCounts;
    const double4* inSlot;
    const uint32_t* inLam;
    const double* cdf;
    SrmChain* chain;     // [B]
};

// Track-length tally of one segment: weight G (e^{gl} - 1)/g split to the
// four corners by the midpoint barycentric weights, added to the ray's
// pending corner tallies.  Returns false (ray dropped) when the contribution
// is not finite.
__device__ __forceinline__ bool tallySegment(const TetView& m, FwdRay& r, double len, const double lam[4],
                                             const double dl[4]) {
    const double gc = gainCoefficient(m, r.c, r.sA, r.sE);
    const double gl = gc * len;
    const double E = expm1(gl);
    const double T = fabs(gl) < 1e-8 ? len : E / gc;
    const double contribution = r.G * T;
    if (!isfinite(contribution)) return false;
    double w[4], wsum = 0.0;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        w[f] = fmax(0.0, fma(0.5 * len, dl[f], lam[f]));
        wsum += w[f];
    }
    const bool split = wsum > DBL_EPSILON;
    const double s = split ? contribution / wsum : 0.25 * contribution;
#pragma unroll
    for (int f = 0; f < 4; ++f) r.pv[f] = fma(split ? w[f] : 1.0, s, r.pv[f]);
    r.G = fma(r.G, E, r.G);
    return true;
}

// Moving from the current cell through its face bf into the neighbour entered
// through its face fe (corner-sorted records, material vertices mn): inside
// one material the neighbour's corners other than fe are the old corners
// other than bf, in the same order, so their pending tallies move over and
// only the old corner bf is added to device memory; a change of material
// (gain <-> cladding, other material vertices) adds all four.
template <typename Flush>
__device__ __forceinline__ void carryPending(FwdRay& r, int bf, int fe, uint4 mn, uint32_t Np, Flush&& flush) {
    if ((r.pid.x >= Np) == (mn.x >= Np)) {
        const double s0 = bf == 0 ? r.pv[1] : r.pv[0];
        const double s1 = bf <= 1 ? r.pv[2] : r.pv[1];
        const double s2 = bf <= 2 ? r.pv[3] : r.pv[2];
        const double v = bf == 0 ? r.pv[0] : bf == 1 ? r.pv[1] : bf == 2 ? r.pv[2] : r.pv[3];
        const uint32_t id = bf == 0 ? r.pid.x : bf == 1 ? r.pid.y : bf == 2 ? r.pid.z : r.pid.w;
        r.pv[0] = fe == 0 ? 0.0 : s0;
        r.pv[1] = fe == 1 ? 0.0 : fe == 0 ? s0 : s1;
        r.pv[2] = fe == 2 ? 0.0 : fe < 2 ? s1 : s2;
        r.pv[3] = fe == 3 ? 0.0 : s2;
        if (v != 0.0) flush(id, v);
    } else {
        const uint32_t o[4] = {r.pid.x, r.pid.y, r.pid.z, r.pid.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (r.pv[j] != 0.0) flush(o[j], r.pv[j]);
            r.pv[j] = 0.0;
        }
    }
    r.pid = mn;
}

template <typename Flush>
__device__ __forceinline__ void flushPending(FwdRay& r, Flush&& flush) {
    const uint32_t o[4] = {r.pid.x, r.pid.y, r.pid.z, r.pid.w};
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (r.pv[j] != 0.0) flush(o[j], r.pv[j]);
}

struct FwdLaunch {
    TetView m;
    const double* sigmaA;
    const double* sigmaE;
    uint32_t nL, seed, launch, B, blocksPerBatch;
    double* score;                 // [B][2 Np]
    uint32_t* visits;              // [C]
    uint32_t* dropped;             // [C]
    uint32_t* next;                // [B]: next unclaimed ray index of each batch (zeroed per launch)
    SrmLaunch srm;                 // reflection passes (kernel modes 1 and 2)
    double shift[kMaxBatches];
    uint32_t nb[kMaxBatches];
    uint32_t phase[kMaxBatches];
};

// Source ray i of batch b (ray r = i B + b of this launch).
__device__ __forceinline__ void initSourceRay(const FwdLaunch& L, uint32_t b, uint32_t i, FwdRay& r) {
    const TetView& m = L.m;
    const uint32_t nb = L.nb[b];
    const double t = (double(i) + L.shift[b]) / double(nb) * m.Btot;
    // upper_bound (first cell whose inclusive prefix exceeds t) inside the
    // guide-table bracket of t, widened by one slot on each side for the
    // rounding of j (indexed search, Chen and Asau 1974)
    const double jf = fmin(fmax(t * m.guideScale, 0.0), double(m.K - 1));
    const uint32_t j = uint32_t(jf);
    uint32_t lo = __ldg(m.guide + (j > 0 ? j - 1 : 0));
    uint32_t hi = __ldg(m.guide + min(j + 2, m.K));
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(m.prefix + mid) > t) hi = mid;
        else lo = mid + 1;
    }
    const uint32_t c = lo >= m.C ? m.lastSource : lo;
    const uint32_t ray = i * L.B + b;
    const Philox4 o = philox4x32_10(ray, L.launch, 0u, kTagFwdRay, L.seed, kFwdKeyHi);
    const Philox4 o2 = philox4x32_10(ray, L.launch, 1u, kTagFwdRay, L.seed, kFwdKeyHi);
    const double e0 = -log(unit53(o.x)), e1 = -log(unit53(o.y)), e2 = -log(unit53(o.z)), e3 = -log(unit53(o.w));
    const double esum = e0 + e1 + e2 + e3;
    // exponential k goes to sorted corner k (ascending point index)
    const CellLinks lk = ldLinks(&m.cell[c].nbr);
    const uint4 mv = lk.matv;
    const uint32_t off = mv.x >= m.Np ? m.Np : 0u;
    const uint4 cv = make_uint4(mv.x - off, mv.y - off, mv.z - off, mv.w - off);
    const double* P = m.points;
    const double w0 = e0 / esum, w1 = e1 / esum, w2 = e2 / esum, w3 = e3 / esum;
    r.x = w0 * P[3 * cv.x] + w1 * P[3 * cv.y] + w2 * P[3 * cv.z] + w3 * P[3 * cv.w];
    r.y = w0 * P[3 * cv.x + 1] + w1 * P[3 * cv.y + 1] + w2 * P[3 * cv.z + 1] + w3 * P[3 * cv.w + 1];
    r.z = w0 * P[3 * cv.x + 2] + w1 * P[3 * cv.y + 2] + w2 * P[3 * cv.z + 2] + w3 * P[3 * cv.w + 2];
    const double z = 2.0 * unit53(o2.x) - 1.0;
    double sphi, cphi;
    sincos(kTwoPi * unit53(o2.y), &sphi, &cphi);
    const double rr = sqrt(fmax(0.0, 1.0 - z * z));
    r.ux = rr * cphi;
    r.uy = rr * sphi;
    r.uz = z;
    // wavelength bin: golden-ratio sequence over the batch's ray index, so the
    // bin is independent of the source cell (the CDF strata run in cell order)
    const uint32_t lamIdx = __umulhi(i * kWeylStep + L.phase[b], L.nL);
    r.sA = __ldg(L.sigmaA + lamIdx);
    r.sE = __ldg(L.sigmaE + lamIdx);
    r.G = 1.0;
    r.c = c;
    r.ff = -1;
    r.steps = 0;
    r.pid = mv;
    r.nbr = lk.nbr;
    r.id = ray;
    r.lam = lamIdx;
#pragma unroll
    for (int k = 0; k < 4; ++k) r.pv[k] = 0.0;
}

// Reflected ray i of batch b (ray r = i B + b) of a reflection pass
// (include/kernels/forward/accumulation.hpp:714-810): its face by the
// stratified target (i + shift_b)/N_b W_b in the input reservoir's face-weight
// CDF, its slot by weight among the face's filled slots, started at the face
// centroid along the stored reflected direction with the chain's previous
// total weight / N_b.  Returns false when the face holds no weight.
__device__ __forceinline__ bool initReflectedRay(const FwdLaunch& L, uint32_t b, uint32_t i, FwdRay& r) {
    const SrmLaunch& S = L.srm;
    const double* cb = S.cdf + size_t(b) * S.nF;
    const double t = (double(i) + L.shift[b]) / double(L.nb[b]) * cb[S.nF - 1];
    uint32_t lo = 0, hi = S.nF;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (cb[mid] > t) hi = mid;
        else lo = mid + 1;
    }
    const uint32_t k = min(lo, S.nF - 1);
    const size_t face = size_t(b) * S.nF + k;
    const uint32_t filled = min(S.inCounts[face], S.S);
    if (filled == 0) return false;
    const double4* slots = S.inSlot + face * S.S;
    double slotSum = 0.0;
    for (uint32_t q = 0; q < filled; ++q) slotSum += slots[q].w;
    if (!(slotSum > 0.0)) return false;
    const uint32_t ray = i * L.B + b;
    const Philox4 o = philox4x32_10(ray, L.launch, S.pass << 2, kTagFwdRay, L.seed, kFwdKeyHi);
    const double target = unit53(o.x) * slotSum;
    double cum = 0.0;
    uint32_t slot = filled - 1;
    for (uint32_t q = 0; q < filled; ++q) {
        cum += slots[q].w;
        if (cum >= target) {
            slot = q;
            break;
        }
    }
    const double4 sd = slots[slot];
    const double len = sqrt(sd.x * sd.x + sd.y * sd.y + sd.z * sd.z);
    const double inv = len > DBL_EPSILON ? 1.0 / len : 0.0;
    r.ux = sd.x * inv;
    r.uy = sd.y * inv;
    r.uz = sd.z * inv;
    const uint32_t lam = S.inLam[face * S.S + slot];
    const BFace& f = S.faces[k];
    r.x = f.cen[0];
    r.y = f.cen[1];
    r.z = f.cen[2];
    r.c = f.c;
    r.ff = int(f.f);
    r.G = S.chain[b].prev / double(L.nb[b]);
    r.sA = __ldg(L.sigmaA + lam);
    r.sE = __ldg(L.sigmaE + lam);
    r.lam = lam;
    r.id = ray;
    r.steps = 0;
    const CellLinks lk = ldLinks(&L.m.cell[r.c].nbr);
    r.pid = lk.matv;
    r.nbr = lk.nbr;
#pragma unroll
    for (int q = 0; q < 4; ++q) r.pv[q] = 0.0;
    return true;
}

// A ray of batch b that left the mesh through reflecting face k: weight x
// gain x reflectance (include/kernels/reflection.hpp:21-47) into the face's
// weighted reservoir of reflected directions
// (include/kernels/forward/accumulation.hpp:455-506).  Slots fill in arrival
// order; once full, a deposit replaces a random slot with probability
// min(1, S w / (W_prior + w)).
__device__ __forceinline__ void depositReflection(const FwdLaunch& L, uint32_t b, uint32_t k, const FwdRay& r) {
    const SrmLaunch& S = L.srm;
    if (S.S == 0 || !(r.G > 0.0) || !isfinite(r.G)) return;
    const BFace& f = S.faces[k];
    const double dn = r.ux * f.n[0] + r.uy * f.n[1] + r.uz * f.n[2];
    const double cosI = fmin(1.0, fabs(dn));
    const double sin2 = fmax(0.0, 1.0 - cosI * cosI);
    const double refl = (f.ratio2 > 0.0 && f.ratio2 * sin2 > 1.0) ? 1.0 : fmax(0.0, f.R);
    const double w = r.G * refl;
    if (!(w > 0.0) || !isfinite(w)) return;
    const size_t face = size_t(b) * S.nF + k;
    const uint32_t seen = atomicAdd(S.outCounts + face, 1u);
    const double prior = atomicAdd(S.outFaceW + face, w);
    uint32_t slot = seen;
    if (slot >= S.S) {
        const Philox4 o = philox4x32_10(r.id, L.launch, (S.pass << 2) | 2u, kTagFwdRay, L.seed, kFwdKeyHi);
        const double p = fmin(1.0, double(S.S) * w / (prior + w));
        if (unit53(o.x) >= p) return;
        slot = min(S.S - 1, uint32_t(unit53(o.y) * double(S.S)));
    }
    double rx = r.ux - f.n[0] * (2.0 * dn), ry = r.uy - f.n[1] * (2.0 * dn), rz = r.uz - f.n[2] * (2.0 * dn);
    const double rl = sqrt(rx * rx + ry * ry + rz * rz);
    const double inv = rl > DBL_EPSILON ? 1.0 / rl : 0.0;
    S.outSlot[face * S.S + slot] = make_double4(rx * inv, ry * inv, rz * inv, w);
    S.outLam[face * S.S + slot] = r.lam;
    S.outRay[face * S.S + slot] = r.id;
}

}  // namespace

namespace {

// Block j serves batch j % B; the blocksPerBatch blocks of a batch stride its
// rays.  SMEM: the block's vertex tallies go to a shared-memory histogram of
// 2 Np doubles, added to the batch's device-memory tallies once at the end.
// MODE 0: source rays; 1: source rays that deposit at reflecting faces (the
// first pass of the surface-reservoir method); 2: reflected rays drawn from
// the reservoir, depositing in turn (blocks of a batch whose chain has ended
// return at once).
template <bool SMEM, int MODE>
__global__ void __launch_bounds__(kFwdBlock, kFwdMinBlocks) fwdRayKernel(const FwdLaunch L) {
    extern __shared__ double hist[];
    const TetView& m = L.m;
    const uint32_t b = blockIdx.x % L.B;
    if (MODE == 2 && !L.srm.chain[b].active) return;
    const uint32_t nV = 2u * m.Np;
    double* gscore = L.score + size_t(b) * nV;
    if (SMEM) {
        for (uint32_t k = threadIdx.x; k < nV; k += blockDim.x) hist[k] = 0.0;
        __syncthreads();
    }
    // Rays of the batch are claimed dynamically: a warp whose idle lanes
    // reach kFwdRefill (or that has no lane walking) takes the next
    // popc(idle) ray indices of its batch with one atomic and starts them
    // together, so every lane of every warp of the batch stays busy until the
    // batch runs dry.
    const uint32_t nb = L.nb[b];
    const int lane = threadIdx.x & 31;
    auto add = [&](uint32_t v, double val) {
        if (SMEM) atomicAdd(hist + v, val);
        else atomicAdd(gscore + v, val);
    };
    FwdRay r;
    bool live = false;
    bool exhausted = nb == 0;  // warp-uniform
    for (;;) {
        const unsigned walking = __ballot_sync(0xffffffffu, live);
        if (walking == 0 && exhausted) break;
        const unsigned idle = ~walking;
        if (!exhausted && idle != 0 && (__popc(idle) >= kFwdRefill || walking == 0)) {
            const int leader = __ffs(idle) - 1;
            const uint32_t want = uint32_t(__popc(idle));
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(L.next + b, want);
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base + want >= nb) exhausted = true;
            if (!live) {
                const uint32_t i = base + uint32_t(__popc(idle & ((1u << lane) - 1u)));
                if (i < nb) {
                    if (MODE == 2) {
                        live = initReflectedRay(L, b, i, r);
                    } else {
                        initSourceRay(L, b, i, r);
                        live = true;
                    }
                }
            }
        }
        // up to kFwdSteps cells per lane before the warp meets again to claim rays
#pragma unroll 1
        for (int k = 0; k < kFwdSteps && live; ++k) {
            double lam[4], dl[4], len;
            const int bf = exitFace(m.cell[r.c].plane, r.x, r.y, r.z, r.ux, r.uy, r.uz, r.ff, lam, dl, len);
            bool drop = bf < 0 || ++r.steps > kFwdMaxSteps;
            const int n = bf == 0 ? r.nbr.x : bf == 1 ? r.nbr.y : bf == 2 ? r.nbr.z : r.nbr.w;
            if (!drop) {
                drop = !tallySegment(m, r, len, lam, dl);
                if (!drop) atomicAdd(L.visits + r.c, 1u);
            }
            if (drop) {
                atomicAdd(L.dropped + r.c, 1u);
                flushPending(r, add);
                live = false;
                break;
            }
            r.x = fma(r.ux, len, r.x);
            r.y = fma(r.uy, len, r.y);
            r.z = fma(r.uz, len, r.z);
            if (n < 0) {
                flushPending(r, add);
                if (MODE != 0 && n <= -2) depositReflection(L, b, uint32_t(-2 - n), r);
                live = false;  // left the mesh
            } else {
                r.c = uint32_t(n) >> 2;
                r.ff = n & 3;
                const CellLinks lk = ldLinks(&m.cell[r.c].nbr);
                r.nbr = lk.nbr;
                carryPending(r, bf, r.ff, lk.matv, m.Np, add);
            }
        }
    }
    if (SMEM) {
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < nV; k += blockDim.x) {
            const double v = hist[k];
            if (v != 0.0) atomicAdd(gscore + k, v);
        }
    }
}

struct FinLaunch {
    const double* score;   // [B][2 Np]
    const double* lumped;  // [2 Np]
    const double* vol;     // [C]
    const double* beta;    // [C] (dndt)
    const TetCell* cell;   // [C] (material vertices)
    const uint32_t* dropped;
    const uint32_t* visits;
    unsigned long long* crossings;  // sum of visits (zeroed before the launch)
    float* phi;
    double* rse;
    double* dndt;
    uint32_t* unconverged;
    uint32_t C, Np, B;
    double Btot, totalRays, nTot, tau, threshold, dndtA, dndtE;
    double raysInBatch[kMaxBatches];
};

// Vertex -> cell density through lumped material-vertex volumes, estimate,
// batch-mean relative error (include/kernels/forwardPhiAseMapping.hpp:51-150).
__global__ void __launch_bounds__(256) fwdFinalizeKernel(const FinLaunch F) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long nvis = c < F.C ? F.visits[c] : 0ull;
    for (int o = 16; o > 0; o >>= 1) nvis += __shfl_xor_sync(0xffffffffu, nvis, o);
    if ((threadIdx.x & 31) == 0 && nvis) atomicAdd(F.crossings, nvis);
    if (c >= F.C) return;
    const uint4 mv = F.cell[c].matv;
    const uint32_t v[4] = {mv.x, mv.y, mv.z, mv.w};
    double lumped[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) lumped[k] = F.lumped[v[k]];
    const double V = F.vol[c];
    const size_t nV = 2u * size_t(F.Np);
    double sum = 0.0, mSum = 0.0, m2Sum = 0.0;
    uint32_t active = 0;
    for (uint32_t b = 0; b < F.B; ++b) {
        double dens = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) dens += lumped[k] > 0.0 ? F.score[b * nV + v[k]] / lumped[k] : 0.0;
        const double bs = dens / 4.0 * V;
        sum += bs;
        if (F.raysInBatch[b] == 0.0) continue;
        const double mean = bs / F.raysInBatch[b];
        mSum += mean;
        m2Sum += mean * mean;
        ++active;
    }
    const double estimate = sum * F.Btot / (F.totalRays * V);
    double rse = DBL_MAX;
    if (F.dropped[c] == 0 && active >= 2) {
        const double mean = mSum / active;
        if (mean == 0.0) {
            rse = nan("");
        } else {
            const double var = fmax(0.0, (m2Sum - mSum * mSum / active) / (active - 1.0));
            rse = sqrt(var / active) / fabs(mean);
        }
    }
    const float phi = __double2float_rn(estimate * F.nTot / F.tau);
    F.phi[c] = phi;
    F.rse[c] = rse;
    F.dndt[c] = (F.beta[c] * (F.dndtE + F.dndtA) - F.dndtA) * double(phi);
    if (!(isfinite(rse) && rse <= F.threshold)) atomicAdd(F.unconverged, 1u);
}

// Inclusive CDF of one batch's reservoir face weights (one block per batch,
// FP64 block scan in chunks of the block size).
constexpr uint32_t kScanBlock = 1024u;
__global__ void __launch_bounds__(kScanBlock) srmScanKernel(const double* faceW, double* cdf, uint32_t nF) {
    __shared__ double warpTot[kScanBlock / 32];
    const double* in = faceW + size_t(blockIdx.x) * nF;
    double* out = cdf + size_t(blockIdx.x) * nF;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double carry = 0.0;
    for (uint32_t base = 0; base < nF; base += kScanBlock) {
        const uint32_t k = base + threadIdx.x;
        double v = k < nF ? in[k] : 0.0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double n = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += n;
        }
        if (lane == 31) warpTot[warp] = v;
        __syncthreads();
        if (warp == 0) {
            double t = warpTot[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double n = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += n;
            }
            warpTot[lane] = t;
        }
        __syncthreads();
        if (warp > 0) v += warpTot[warp - 1];
        if (k < nF) out[k] = carry + v;
        carry += warpTot[kScanBlock / 32 - 1];
        __syncthreads();
    }
}

// Slots in ray order: a face that received no more deposits than it has
// slots holds every deposit, in the order the atomics happened to assign;
// sorting them by ray index makes the reservoir (and so the next pass's
// reflected rays) independent of that order.  Faces that overflowed keep the
// slots their random replacements chose.  One thread per (batch, face).
__global__ void srmSortKernel(const uint32_t* counts, double4* slot, uint32_t* lam, uint32_t* ray, uint32_t S,
                              size_t faces) {
    const size_t face = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (face >= faces) return;
    const uint32_t n = counts[face];
    if (n < 2 || n > S) return;
    double4* sl = slot + face * S;
    uint32_t* la = lam + face * S;
    uint32_t* ra = ray + face * S;
    for (uint32_t i = 1; i < n; ++i) {
        const double4 v = sl[i];
        const uint32_t l = la[i], r = ra[i];
        uint32_t j = i;
        while (j > 0 && ra[j - 1] > r) {
            sl[j] = sl[j - 1];
            la[j] = la[j - 1];
            ra[j] = ra[j - 1];
            --j;
        }
        sl[j] = v;
        la[j] = l;
        ra[j] = r;
    }
}

// Status of every batch's chain after a pass (include/core/forwardSrm.hpp:
// 281-363): pass 0 opens the chain with the first reservoir's weight (none:
// converged); later passes compare the new total weight with the previous
// one: a growth streak of `streak` passes ends it as diverged, a relative
// change below `tol` as stable, a weight below tol x the first as converged.
__global__ void srmControlKernel(SrmChain* chain, const double* cdf, uint32_t nF, uint32_t B, uint32_t pass,
                                 double tol, uint32_t streak) {
    const uint32_t b = threadIdx.x;
    if (b >= B) return;
    const double cur = nF ? cdf[size_t(b) * nF + nF - 1] : 0.0;
    SrmChain& ch = chain[b];
    if (pass == 0) {
        ch.grow = 0;
        ch.passes = 0;
        if (cur == 0.0) {
            ch.initial = ch.prev = ch.remaining = 0.0;
            ch.status = kSrmConverged;
            ch.active = 0;
        } else {
            ch.initial = ch.prev = cur;
            ch.remaining = 1.0;
            ch.status = kSrmMaxIterations;
            ch.active = 1;
        }
        return;
    }
    if (!ch.active) return;
    ch.passes = pass;
    ch.remaining = cur / ch.initial;
    if (cur > ch.prev) {
        if (++ch.grow >= streak) {
            ch.status = kSrmDiverged;
            ch.active = 0;
            return;
        }
    } else {
        ch.grow = 0;
        if (fabs(cur - ch.prev) / fmax(cur, 1.0e-30) < tol) {
            ch.status = kSrmStable;
            ch.active = 0;
            return;
        }
    }
    if (ch.remaining < tol) {
        ch.status = kSrmConverged;
        ch.active = 0;
        return;
    }
    ch.prev = cur;
}

struct TraceLaunch {
    TetView m;
    uint32_t n, maxSegments;
    const uint32_t* startCell;
    const double* origin;
    const double* direction;
    double sA, sE;
    uint32_t* segments;
    uint32_t* cells;
    double* lengths;
    double* lnGain;
    double* endPoint;
    int32_t* status;
};

__global__ void __launch_bounds__(128) fwdTraceKernel(const TraceLaunch T) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.n) return;
    const TetView& m = T.m;
    FwdRay r;
    r.x = T.origin[3 * size_t(i)];
    r.y = T.origin[3 * size_t(i) + 1];
    r.z = T.origin[3 * size_t(i) + 2];
    r.ux = T.direction[3 * size_t(i)];
    r.uy = T.direction[3 * size_t(i) + 1];
    r.uz = T.direction[3 * size_t(i) + 2];
    r.c = T.startCell[i];
    r.ff = -1;
    r.steps = 0;
    double lg = 0.0;
    int32_t st = 1;
    uint32_t seg = 0;
    while (seg < uint32_t(kFwdMaxSteps)) {
        double lam[4], dl[4], len;
        const TetCell* rec = m.cell + r.c;
        const int bf = exitFace(rec->plane, r.x, r.y, r.z, r.ux, r.uy, r.uz, r.ff, lam, dl, len);
        if (bf < 0) break;
        lg += gainCoefficient(m, r.c, T.sA, T.sE) * len;
        if (seg < T.maxSegments) {
            if (T.cells) T.cells[size_t(i) * T.maxSegments + seg] = r.c;
            if (T.lengths) T.lengths[size_t(i) * T.maxSegments + seg] = len;
        }
        ++seg;
        r.x = fma(r.ux, len, r.x);
        r.y = fma(r.uy, len, r.y);
        r.z = fma(r.uz, len, r.z);
        const int n = (&rec->nbr.x)[bf];
        if (n < 0) {
            st = 0;
            break;
        }
        r.c = uint32_t(n) >> 2;
        r.ff = n & 3;
    }
    T.segments[i] = seg;
    T.lnGain[i] = lg;
    T.endPoint[3 * size_t(i)] = r.x;
    T.endPoint[3 * size_t(i) + 1] = r.y;
    T.endPoint[3 * size_t(i) + 2] = r.z;
    T.status[i] = st;
}

}  // namespace

// ------------------------------------------------------------ host side ----
namespace {

struct TetHost {
    std::vector<double4> plane;
    std::vector<int> nbr;
    std::vector<uint4> matv;
    std::vector<double> vol, lumped;
};

// Barycentric face planes, volumes and face neighbours of a Tet4 mesh.  Face f
// of a cell is opposite its vertex f; lambda_f = delta_f0 + grad_f . (x - v0)
// with grad_1..3 the rows of E^-1 (E = [v1-v0, v2-v0, v3-v0]) and grad_0 =
// -(grad_1 + grad_2 + grad_3), stored as planes a.x + d.
hase_status buildTetHost(const hase_tet_mesh_desc* d, TetHost& h) {
    const uint32_t C = d->numberOfCells, Np = d->numberOfPoints;
    h.plane.resize(4 * size_t(C));
    h.nbr.assign(4 * size_t(C), -1);
    h.matv.resize(C);
    h.vol.resize(C);
    h.lumped.assign(2 * size_t(Np), 0.0);
    struct FaceKey {
        uint32_t a, b, c, id;
    };
    std::vector<FaceKey> faces(4 * size_t(C));
    for (uint32_t c = 0; c < C; ++c) {
        const uint32_t* v = d->cells + 4 * size_t(c);
        for (int k = 0; k < 4; ++k)
            if (v[k] >= Np) return fail(HASE_INVALID_ARGUMENT, "cell %u references point %u >= %u", c, v[k], Np);
        const double* p0 = d->points + 3 * size_t(v[0]);
        double E[3][3];
        for (int k = 1; k < 4; ++k)
            for (int a = 0; a < 3; ++a) E[a][k - 1] = d->points[3 * size_t(v[k]) + a] - p0[a];
        const double det = E[0][0] * (E[1][1] * E[2][2] - E[1][2] * E[2][1]) -
                           E[0][1] * (E[1][0] * E[2][2] - E[1][2] * E[2][0]) +
                           E[0][2] * (E[1][0] * E[2][1] - E[1][1] * E[2][0]);
        if (!(std::fabs(det) > 0.0) || !std::isfinite(det))
            return fail(HASE_INVALID_ARGUMENT, "cell %u is degenerate", c);
        h.vol[c] = std::fabs(det) / 6.0;
        double inv[3][3];
        inv[0][0] = (E[1][1] * E[2][2] - E[1][2] * E[2][1]) / det;
        inv[0][1] = (E[0][2] * E[2][1] - E[0][1] * E[2][2]) / det;
        inv[0][2] = (E[0][1] * E[1][2] - E[0][2] * E[1][1]) / det;
        inv[1][0] = (E[1][2] * E[2][0] - E[1][0] * E[2][2]) / det;
        inv[1][1] = (E[0][0] * E[2][2] - E[0][2] * E[2][0]) / det;
        inv[1][2] = (E[0][2] * E[1][0] - E[0][0] * E[1][2]) / det;
        inv[2][0] = (E[1][0] * E[2][1] - E[1][1] * E[2][0]) / det;
        inv[2][1] = (E[0][1] * E[2][0] - E[0][0] * E[2][1]) / det;
        inv[2][2] = (E[0][0] * E[1][1] - E[0][1] * E[1][0]) / det;
        double g[4][3];
        for (int a = 0; a < 3; ++a) {
            g[1][a] = inv[0][a];
            g[2][a] = inv[1][a];
            g[3][a] = inv[2][a];
            g[0][a] = -(inv[0][a] + inv[1][a] + inv[2][a]);
        }
        for (int f = 0; f < 4; ++f) {
            const double dd = (f == 0 ? 1.0 : 0.0) - (g[f][0] * p0[0] + g[f][1] * p0[1] + g[f][2] * p0[2]);
            h.plane[4 * size_t(c) + f] = make_double4(g[f][0], g[f][1], g[f][2], dd);
        }
        const bool clad = d->claddingCellTypes && d->claddingCellTypes[c] == d->claddingNumber;
        const uint32_t off = clad ? Np : 0u;
        h.matv[c] = make_uint4(v[0] + off, v[1] + off, v[2] + off, v[3] + off);
        for (int k = 0; k < 4; ++k) h.lumped[v[k] + off] += h.vol[c] / 4.0;
        for (int f = 0; f < 4; ++f) {
            uint32_t a[3], n = 0;
            for (int k = 0; k < 4; ++k)
                if (k != f) a[n++] = v[k];
            std::sort(a, a + 3);
            faces[4 * size_t(c) + f] = FaceKey{a[0], a[1], a[2], uint32_t(4 * c + f)};
        }
    }
    std::sort(faces.begin(), faces.end(), [](const FaceKey& x, const FaceKey& y) {
        return std::tie(x.a, x.b, x.c, x.id) < std::tie(y.a, y.b, y.c, y.id);
    });
    auto same = [](const FaceKey& x, const FaceKey& y) { return x.a == y.a && x.b == y.b && x.c == y.c; };
    for (size_t k = 0; k < faces.size();) {
        size_t e = k + 1;
        while (e < faces.size() && same(faces[k], faces[e])) ++e;
        if (e - k > 2) return fail(HASE_INVALID_ARGUMENT, "a face is shared by more than two cells");
        if (e - k == 2) {
            const uint32_t x = faces[k].id, y = faces[k + 1].id;
            h.nbr[x] = int(y);  // ids are 4 * cell + face = the packed (cell << 2) | face
            h.nbr[y] = int(x);
        }
        k = e;
    }
    return HASE_OK;
}

uint32_t forwardTarget(uint32_t minRays, uint32_t maxRays, uint32_t steps, uint32_t k) {
    // include/core/types.hpp:333-354: geometric growth minRays -> maxRays in `steps` increases.
    if (maxRays <= minRays || steps == 0) return minRays;
    if (k >= steps) return maxRays;
    const double growth = std::pow(double(maxRays) / double(minRays), 1.0 / double(steps));
    const uint32_t r = uint32_t(std::ceil(double(minRays) * std::pow(growth, double(k))));
    return std::min(std::max(r, minRays), maxRays);
}

}  // namespace

struct hase_tet_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    uint32_t C = 0, Np = 0, lastSource = 0, numSMs = 0;
    double nTot = 0, tau = 0, cladAbs = 0, Btot = 0;
    uint32_t cladNumber = 0;
    std::vector<uint32_t> cladTypes;
    std::vector<double> vol, sigmaA, sigmaE;
    DevBuf<TetCell> cell;
    std::vector<uint8_t> sortedCorner;  // [C][4]: caller's corner index of sorted corner k
    DevBuf<uint32_t> guide;
    uint32_t K = 1;
    double guideScale = 0.0;
    DevBuf<double> gainBeta, beta, points, prefix, lumped, dvol, sigA, sigE;
    // accumulators and outputs
    DevBuf<double> score, rse, dndt;
    DevBuf<uint32_t> visits, dropped, unconverged, next;
    DevBuf<unsigned long long> crossings;
    DevBuf<float> phi;
    // reflecting boundary faces and the surface-reservoir workspace (two reservoirs)
    DevBuf<BFace> bfaces;
    uint32_t nBF = 0;
    DevBuf<uint32_t> resCounts[2], resLam[2], resRay[2];
    DevBuf<double> resW[2], cdf;
    DevBuf<double4> resSlot[2];
    DevBuf<SrmChain> chain;

    TetView view() const {
        TetView v{};
        v.cell = cell.p;
        v.gainBeta = gainBeta.p;
        v.points = points.p;
        v.prefix = prefix.p;
        v.guide = guide.p;
        v.C = C;
        v.Np = Np;
        v.lastSource = lastSource;
        v.K = K;
        v.guideScale = guideScale;
        v.cladAbs = cladAbs;
        v.nTot = nTot;
        v.Btot = Btot;
        return v;
    }
};

namespace {

hase_status uploadTetBeta(hase_tet_context* c, const double* betaVolume) {
    std::vector<double> gain(c->C), pre(c->C);
    double acc = 0.0;
    uint32_t last = 0;
    for (uint32_t k = 0; k < c->C; ++k) {
        const double b = betaVolume[k];
        if (!std::isfinite(b)) return fail(HASE_INVALID_ARGUMENT, "betaVolume[%u] is not finite", k);
        const bool clad = !c->cladTypes.empty() && c->cladTypes[k] == c->cladNumber;
        gain[k] = clad ? NAN : b;
        const double w = b * c->vol[k];
        if (w < 0.0) return fail(HASE_INVALID_ARGUMENT, "betaVolume[%u] is negative", k);
        acc += w;
        pre[k] = acc;
        if (w > 0.0) last = k;
    }
    c->Btot = acc;
    c->lastSource = last;
    // guide table of the source CDF: guide[j] = upper_bound(prefix, j Btot / K)
    const uint32_t K = c->C;
    std::vector<uint32_t> guide(size_t(K) + 1);
    uint32_t at = 0;
    for (uint32_t j = 0; j < K; ++j) {
        const double bj = double(j) * (acc / double(K));
        while (at < c->C && !(pre[at] > bj)) ++at;
        guide[j] = at;
    }
    guide[K] = c->C;
    c->K = K;
    c->guideScale = acc > 0.0 ? double(K) / acc : 0.0;
    HASE_CUDA(cudaMemcpyAsync(c->guide.p, guide.data(), guide.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                              c->stream));
    HASE_CUDA(cudaMemcpyAsync(c->gainBeta.p, gain.data(), c->C * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    HASE_CUDA(cudaMemcpyAsync(c->beta.p, betaVolume, c->C * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    HASE_CUDA(cudaMemcpyAsync(c->prefix.p, pre.data(), c->C * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    HASE_CUDA(cudaStreamSynchronize(c->stream));
    return HASE_OK;
}

template <typename T>
hase_status upload(DevBuf<T>& buf, const T* src, size_t n, cudaStream_t s) {
    HASE_CUDA(buf.ensure(n));
    HASE_CUDA(cudaMemcpyAsync(buf.p, src, n * sizeof(T), cudaMemcpyHostToDevice, s));
    return HASE_OK;
}

hase_status requireDevice(int device) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(HASE_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= count) return fail(HASE_INVALID_ARGUMENT, "device %d out of range", device);
    return HASE_OK;
}

}  // namespace

extern "C" {

hase_status hase_tet_context_create(const hase_tet_mesh_desc* d, const hase_spectrum_desc* sp, int device,
                                    hase_tet_context** out) {
    if (!d || !sp || !out) return fail(HASE_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (d->numberOfCells == 0 || d->numberOfPoints < 4) return fail(HASE_INVALID_ARGUMENT, "empty mesh");
    if (d->numberOfCells >= (1u << 29)) return fail(HASE_INVALID_ARGUMENT, "mesh too large (at most 2^29 cells)");
    if (d->numberOfPoints >= (1u << 30)) return fail(HASE_INVALID_ARGUMENT, "mesh too large (at most 2^30 points)");
    if (!d->points || !d->cells || !d->betaVolume) return fail(HASE_INVALID_ARGUMENT, "mesh arrays missing");
    if (!(d->nTot > 0.0) || !(d->crystalTFluo > 0.0))
        return fail(HASE_INVALID_ARGUMENT, "nTot and crystalTFluo must be positive");
    if (!std::isfinite(d->claddingAbsorption)) return fail(HASE_INVALID_ARGUMENT, "claddingAbsorption is not finite");
    if (sp->numberOfWavelengths == 0 || !sp->sigmaA || !sp->sigmaE) return fail(HASE_INVALID_ARGUMENT, "empty spectrum");
    for (uint32_t l = 0; l < sp->numberOfWavelengths; ++l)
        if (!std::isfinite(sp->sigmaA[l]) || !std::isfinite(sp->sigmaE[l]))
            return fail(HASE_INVALID_ARGUMENT, "cross section %u is not finite", l);
    for (size_t k = 0; k < 3 * size_t(d->numberOfPoints); ++k)
        if (!std::isfinite(d->points[k])) return fail(HASE_INVALID_ARGUMENT, "point coordinates must be finite");
    HASE_TRY(requireDevice(device));

    TetHost h;
    HASE_TRY(buildTetHost(d, h));
    hase_tet_context* c = new (std::nothrow) hase_tet_context();
    if (!c) return fail(HASE_OUT_OF_MEMORY, "host allocation failed");
    auto cleanup = [&](hase_status s) {
        hase_tet_context_destroy(c);
        return s;
    };
    c->device = device;
    c->C = d->numberOfCells;
    c->Np = d->numberOfPoints;
    c->nTot = d->nTot;
    c->tau = d->crystalTFluo;
    c->cladAbs = d->claddingAbsorption;
    c->cladNumber = d->claddingNumber;
    if (d->claddingCellTypes) c->cladTypes.assign(d->claddingCellTypes, d->claddingCellTypes + c->C);
    c->vol = h.vol;
    c->sigmaA.assign(sp->sigmaA, sp->sigmaA + sp->numberOfWavelengths);
    c->sigmaE.assign(sp->sigmaE, sp->sigmaE + sp->numberOfWavelengths);
    if (cudaSetDevice(device) != cudaSuccess) return cleanup(fail(HASE_CUDA_ERROR, "cudaSetDevice failed"));
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return cleanup(fail(HASE_CUDA_ERROR, "cannot query the SM count"));
    c->numSMs = uint32_t(sms);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev[0]) != cudaSuccess || cudaEventCreate(&c->ev[1]) != cudaSuccess)
        return cleanup(fail(HASE_CUDA_ERROR, "stream/event creation failed"));
    const size_t C = c->C, Np = c->Np;
    hase_status st = HASE_OK;
    // corner-sorted records: sorted corner k is the caller's corner srt[k];
    // the face opposite it keeps its plane, its neighbour gets the
    // neighbour's sorted face index
    c->sortedCorner.resize(4 * C);
    std::vector<uint8_t> inv(4 * C);
    for (size_t k = 0; k < C; ++k) {
        uint8_t srt[4] = {0, 1, 2, 3};
        const uint32_t* v = d->cells + 4 * k;
        std::sort(srt, srt + 4, [&](uint8_t a, uint8_t b) { return v[a] < v[b]; });
        for (int j = 0; j < 4; ++j) {
            c->sortedCorner[4 * k + j] = srt[j];
            inv[4 * k + srt[j]] = uint8_t(j);
        }
    }
    std::vector<TetCell> rec(C);
    for (size_t k = 0; k < C; ++k) {
        const uint8_t* srt = &c->sortedCorner[4 * k];
        for (int j = 1; j < 4; ++j) rec[k].plane[j - 1] = h.plane[4 * k + srt[j]];
        int n4[4];
        uint32_t mv[4];
        const uint32_t hm[4] = {h.matv[k].x, h.matv[k].y, h.matv[k].z, h.matv[k].w};
        for (int j = 0; j < 4; ++j) {
            const int id = h.nbr[4 * k + srt[j]];
            n4[j] = id < 0 ? -1 : int((uint32_t(id) >> 2) << 2 | inv[4 * (size_t(id) >> 2) + (id & 3)]);
            mv[j] = hm[srt[j]];
        }
        rec[k].nbr = make_int4(n4[0], n4[1], n4[2], n4[3]);
        rec[k].matv = make_uint4(mv[0], mv[1], mv[2], mv[3]);
    }
    // reflecting boundary faces: outward normal of the face's points turned
    // away from the cell centre (include/kernels/forward/rayWalk.hpp:60-84),
    // centroid, reflectivity and index ratio resolved as
    // include/core/mesh.hpp:301-332; the record's neighbour code -2 - k
    std::vector<BFace> bf;
    if (d->cellFaceBoundaries) {
        for (size_t k = 0; k < C; ++k) {
            const uint32_t* v = d->cells + 4 * k;
            for (int f = 0; f < 4; ++f) {
                const int32_t id = d->cellFaceBoundaries[4 * k + f];
                if (h.nbr[4 * k + f] >= 0 || id <= 0) continue;
                BFace b{};
                const double* P[3];
                int n = 0;
                for (int j = 0; j < 4; ++j)
                    if (j != f) P[n++] = d->points + 3 * size_t(v[j]);
                double e1[3], e2[3], cc[3] = {0, 0, 0};
                for (int a = 0; a < 3; ++a) {
                    e1[a] = P[1][a] - P[0][a];
                    e2[a] = P[2][a] - P[0][a];
                    b.cen[a] = (P[0][a] + P[1][a] + P[2][a]) / 3.0;
                    for (int j = 0; j < 4; ++j) cc[a] += d->points[3 * size_t(v[j]) + a] / 4.0;
                }
                double nn[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                                e1[0] * e2[1] - e1[1] * e2[0]};
                const double len = std::sqrt(nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2]);
                for (int a = 0; a < 3; ++a) nn[a] /= len;
                if (nn[0] * (cc[0] - b.cen[0]) + nn[1] * (cc[1] - b.cen[1]) + nn[2] * (cc[2] - b.cen[2]) > 0.0)
                    for (int a = 0; a < 3; ++a) nn[a] = -nn[a];
                for (int a = 0; a < 3; ++a) b.n[a] = nn[a];
                const uint32_t sid = uint32_t(id);
                if (d->surfaceReflectivities && sid < d->numberOfSurfaces) b.R = d->surfaceReflectivities[sid];
                else b.R = d->reflectivities ? d->reflectivities[2 * k + f % 2] : 0.0;
                double nIn, nOut;
                if (d->surfaceRefractiveIndexInside && sid < d->numberOfSurfaces)
                    nIn = d->surfaceRefractiveIndexInside[sid];
                else nIn = d->refractiveIndices ? d->refractiveIndices[2 * (f % 2)] : 1.0;
                if (d->surfaceRefractiveIndexOutside && sid < d->numberOfSurfaces)
                    nOut = d->surfaceRefractiveIndexOutside[sid];
                else nOut = d->refractiveIndices ? d->refractiveIndices[2 * (f % 2) + 1] : 1.0;
                if (!std::isfinite(b.R) || !std::isfinite(nIn) || !std::isfinite(nOut))
                    return cleanup(fail(HASE_INVALID_ARGUMENT, "surface of cell %zu face %d is not finite", k, f));
                b.ratio2 = (nIn > 0.0 && nOut > 0.0) ? (nIn / nOut) * (nIn / nOut) : -1.0;
                b.c = uint32_t(k);
                b.f = inv[4 * k + f];
                (&rec[k].nbr.x)[inv[4 * k + f]] = -2 - int(bf.size());
                bf.push_back(b);
            }
        }
        if (bf.size() >= (size_t(1) << 30)) return cleanup(fail(HASE_INVALID_ARGUMENT, "too many reflecting faces"));
    }
    c->nBF = uint32_t(bf.size());
    if (!bf.empty() && (st = upload(c->bfaces, bf.data(), bf.size(), c->stream)) != HASE_OK) return cleanup(st);
    if ((st = upload(c->cell, rec.data(), C, c->stream)) != HASE_OK ||
        (st = upload(c->points, d->points, 3 * Np, c->stream)) != HASE_OK ||
        (st = upload(c->lumped, h.lumped.data(), 2 * Np, c->stream)) != HASE_OK ||
        (st = upload(c->dvol, h.vol.data(), C, c->stream)) != HASE_OK ||
        (st = upload(c->sigA, c->sigmaA.data(), c->sigmaA.size(), c->stream)) != HASE_OK ||
        (st = upload(c->sigE, c->sigmaE.data(), c->sigmaE.size(), c->stream)) != HASE_OK)
        return cleanup(st);
    if (c->gainBeta.ensure(C) != cudaSuccess || c->beta.ensure(C) != cudaSuccess || c->prefix.ensure(C) != cudaSuccess ||
        c->guide.ensure(C + 1) != cudaSuccess)
        return cleanup(fail(HASE_OUT_OF_MEMORY, "device allocation failed"));
    if ((st = uploadTetBeta(c, d->betaVolume)) != HASE_OK) return cleanup(st);
    *out = c;
    return HASE_OK;
}

hase_status hase_tet_context_info(hase_tet_context* c, uint32_t* numberOfCells, uint32_t* numberOfPoints) {
    if (!c) return fail(HASE_INVALID_ARGUMENT, "null context");
    if (numberOfCells) *numberOfCells = c->C;
    if (numberOfPoints) *numberOfPoints = c->Np;
    return HASE_OK;
}

hase_status hase_tet_context_update_beta(hase_tet_context* c, const double* betaVolume) {
    if (!c || !betaVolume) return fail(HASE_INVALID_ARGUMENT, "null argument");
    HASE_CUDA(cudaSetDevice(c->device));
    return uploadTetBeta(c, betaVolume);
}

hase_status hase_tet_context_destroy(hase_tet_context* c) {
    if (!c) return HASE_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (cudaEvent_t& e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return HASE_OK;
}

hase_status hase_tet_tables(hase_tet_context* c, int32_t* neighbors, int32_t* neighborFace, double* planes,
                            double* volumes) {
    if (!c) return fail(HASE_INVALID_ARGUMENT, "null context");
    HASE_CUDA(cudaSetDevice(c->device));
    const size_t C = c->C;
    std::vector<TetCell> rec(C);
    HASE_CUDA(cudaMemcpyAsync(rec.data(), c->cell.p, C * sizeof(TetCell), cudaMemcpyDeviceToHost, c->stream));
    HASE_CUDA(cudaStreamSynchronize(c->stream));
    for (size_t k = 0; k < C; ++k) {
        const int n4[4] = {rec[k].nbr.x, rec[k].nbr.y, rec[k].nbr.z, rec[k].nbr.w};
        const double4 q1 = rec[k].plane[0], q2 = rec[k].plane[1], q3 = rec[k].plane[2];
        const double4 q0 = make_double4(-(q1.x + q2.x + q3.x), -(q1.y + q2.y + q3.y), -(q1.z + q2.z + q3.z),
                                        1.0 - (q1.w + q2.w + q3.w));
        const double4 q[4] = {q0, q1, q2, q3};
        for (int j = 0; j < 4; ++j) {
            const int f = c->sortedCorner[4 * k + j];  // the caller's face index of sorted face j
            const int n = n4[j] < 0 ? -1 : n4[j] >> 2;
            if (neighbors) neighbors[4 * k + f] = n;
            if (neighborFace) neighborFace[4 * k + f] = n < 0 ? -1 : c->sortedCorner[4 * size_t(n) + (n4[j] & 3)];
            if (planes) {
                const double4 p = q[j];
                planes[16 * k + 4 * f] = p.x;
                planes[16 * k + 4 * f + 1] = p.y;
                planes[16 * k + 4 * f + 2] = p.z;
                planes[16 * k + 4 * f + 3] = p.w;
            }
        }
    }
    if (volumes) HASE_CUDA(cudaMemcpyAsync(volumes, c->dvol.p, C * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    HASE_CUDA(cudaStreamSynchronize(c->stream));
    return HASE_OK;
}

hase_status hase_tet_trace(hase_tet_context* c, uint32_t n, const uint32_t* startCell, const double* origin,
                           const double* direction, uint32_t wavelength, uint32_t maxSegments, uint32_t* segments,
                           uint32_t* cells, double* lengths, double* lnGain, double* endPoint, int32_t* status) {
    if (!c || !startCell || !origin || !direction || !segments || !lnGain || !endPoint || !status)
        return fail(HASE_INVALID_ARGUMENT, "null argument");
    if (wavelength >= c->sigmaA.size()) return fail(HASE_INVALID_ARGUMENT, "wavelength index out of range");
    if (n == 0) return HASE_OK;
    for (uint32_t i = 0; i < n; ++i)
        if (startCell[i] >= c->C) return fail(HASE_INVALID_ARGUMENT, "startCell[%u] out of range", i);
    HASE_CUDA(cudaSetDevice(c->device));
    const size_t N = n, S = size_t(n) * maxSegments;
    DevBuf<uint32_t> dStart, dSeg, dCells;
    DevBuf<double> dOrigin, dDir, dLen, dLn, dEnd;
    DevBuf<int32_t> dStatus;
    HASE_TRY(upload(dStart, startCell, N, c->stream));
    HASE_TRY(upload(dOrigin, origin, 3 * N, c->stream));
    HASE_TRY(upload(dDir, direction, 3 * N, c->stream));
    HASE_CUDA(dSeg.ensure(N));
    HASE_CUDA(dLn.ensure(N));
    HASE_CUDA(dEnd.ensure(3 * N));
    HASE_CUDA(dStatus.ensure(N));
    if (cells && S) HASE_CUDA(dCells.ensure(S));
    if (lengths && S) HASE_CUDA(dLen.ensure(S));
    TraceLaunch T{};
    T.m = c->view();
    T.n = n;
    T.maxSegments = maxSegments;
    T.startCell = dStart.p;
    T.origin = dOrigin.p;
    T.direction = dDir.p;
    T.sA = c->sigmaA[wavelength];
    T.sE = c->sigmaE[wavelength];
    T.segments = dSeg.p;
    T.cells = dCells.p;
    T.lengths = dLen.p;
    T.lnGain = dLn.p;
    T.endPoint = dEnd.p;
    T.status = dStatus.p;
    fwdTraceKernel<<<(n + 127) / 128, 128, 0, c->stream>>>(T);
    HASE_CUDA(cudaGetLastError());
    HASE_CUDA(cudaMemcpyAsync(segments, dSeg.p, N * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    HASE_CUDA(cudaMemcpyAsync(lnGain, dLn.p, N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    HASE_CUDA(cudaMemcpyAsync(endPoint, dEnd.p, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    HASE_CUDA(cudaMemcpyAsync(status, dStatus.p, N * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    if (cells && S) HASE_CUDA(cudaMemcpyAsync(cells, dCells.p, S * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    if (lengths && S) HASE_CUDA(cudaMemcpyAsync(lengths, dLen.p, S * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    HASE_CUDA(cudaStreamSynchronize(c->stream));
    return HASE_OK;
}

}  // extern "C"

extern "C" hase_status hase_tet_calc_phi_ase(hase_tet_context* c, const hase_forward_desc* fw,
                                             hase_forward_result* res) {
    if (!c || !fw || !res) return fail(HASE_INVALID_ARGUMENT, "null argument");
    if (fw->forwardRayCount == 0) return fail(HASE_INVALID_ARGUMENT, "forwardRayCount must be positive");
    const uint32_t B = fw->batches ? fw->batches : 8u;
    if (B < 2 || B > kMaxBatches) return fail(HASE_INVALID_ARGUMENT, "batches must be in [2, %u]", kMaxBatches);
    if (!(fw->relativeStandardErrorThreshold >= 0.0))
        return fail(HASE_INVALID_ARGUMENT, "relativeStandardErrorThreshold must be >= 0");
    if (fw->tallyMode > 2) return fail(HASE_INVALID_ARGUMENT, "tallyMode must be 0, 1 or 2");
    const uint32_t block = fw->blockSize ? fw->blockSize : kFwdBlock;
    if (block != kFwdBlock) return fail(HASE_INVALID_ARGUMENT, "blockSize must be 0 or %u", kFwdBlock);
    const uint32_t minRays = fw->forwardRayCount;
    const uint32_t maxRays = std::max(fw->maxRays, minRays);
    const bool adaptive = maxRays > minRays && fw->adaptiveSteps > 0;
    HASE_CUDA(cudaSetDevice(c->device));

    const uint32_t C = c->C, Np = c->Np;
    const size_t nV = 2 * size_t(Np);
    const size_t histBytes = nV * sizeof(double);
    bool smem = fw->tallyMode == 2 || (fw->tallyMode == 0 && histBytes <= kMaxHistogramBytes);
    if (smem && histBytes > kMaxHistogramBytes)
        return fail(HASE_INVALID_ARGUMENT, "shared-memory tallies need 2 * numberOfPoints * 8 <= %zu bytes",
                    kMaxHistogramBytes);
    int perSM = 0;
    const bool srm = fw->useReflections != 0;
    if (smem) {
        HASE_CUDA(cudaFuncSetAttribute(fwdRayKernel<true, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(histBytes)));
        HASE_CUDA(cudaFuncSetAttribute(fwdRayKernel<true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(histBytes)));
        HASE_CUDA(cudaFuncSetAttribute(fwdRayKernel<true, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(histBytes)));
        HASE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fwdRayKernel<true, 0>, block, histBytes));
    } else {
        HASE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fwdRayKernel<false, 0>, block, 0));
    }
    // surface-reservoir controls (include/core/types.hpp:328-330, src/core/srm.cpp:36-41)
    const uint32_t srmMaxIt = fw->reflectionMaxIterations ? fw->reflectionMaxIterations : 40u;
    const double srmTol = fw->reflectionTolerance > 0.0 ? fw->reflectionTolerance : 1.0e-4;
    const uint32_t srmSlots = fw->surfaceReservoirSize ? fw->surfaceReservoirSize : 32u;
    const uint32_t srmStreak = fw->divergenceStreak ? fw->divergenceStreak : 3u;
    if (srm && !(std::isfinite(fw->reflectionTolerance) && fw->reflectionTolerance >= 0.0))
        return fail(HASE_INVALID_ARGUMENT, "reflectionTolerance must be >= 0");
    if (srm && srmSlots > 4096) return fail(HASE_INVALID_ARGUMENT, "surfaceReservoirSize must be <= 4096");
    const uint32_t nF = c->nBF;
    if (srm && nF > 0) {
        const size_t faces = size_t(B) * nF, slots = faces * srmSlots;
        for (int k = 0; k < 2; ++k) {
            HASE_CUDA(c->resCounts[k].ensure(faces));
            HASE_CUDA(c->resW[k].ensure(faces));
            HASE_CUDA(c->resSlot[k].ensure(slots));
            HASE_CUDA(c->resLam[k].ensure(slots));
            HASE_CUDA(c->resRay[k].ensure(slots));
        }
        HASE_CUDA(c->cdf.ensure(faces));
        HASE_CUDA(c->chain.ensure(B));
    }
    if (perSM < 1) return fail(HASE_CUDA_ERROR, "the ray kernel does not fit on an SM");
    const uint32_t resident = uint32_t(perSM) * c->numSMs;

    HASE_CUDA(c->score.ensure(size_t(B) * nV));
    HASE_CUDA(c->visits.ensure(C));
    HASE_CUDA(c->dropped.ensure(C));
    HASE_CUDA(c->unconverged.ensure(1));
    HASE_CUDA(c->next.ensure(kMaxBatches));
    HASE_CUDA(c->crossings.ensure(1));
    HASE_CUDA(c->phi.ensure(C));
    HASE_CUDA(c->rse.ensure(C));
    HASE_CUDA(c->dndt.ensure(C));
    HASE_CUDA(cudaMemsetAsync(c->score.p, 0, size_t(B) * nV * sizeof(double), c->stream));
    HASE_CUDA(cudaMemsetAsync(c->visits.p, 0, C * sizeof(uint32_t), c->stream));
    HASE_CUDA(cudaMemsetAsync(c->dropped.p, 0, C * sizeof(uint32_t), c->stream));
    HASE_CUDA(cudaMemsetAsync(c->crossings.p, 0, sizeof(unsigned long long), c->stream));

    const uint32_t nL = fw->monochromatic ? 1u : uint32_t(c->sigmaA.size());
    double dA = c->sigmaA[0], dE = c->sigmaE[0];
    if (nL > 1)
        for (uint32_t l = 1; l < nL; ++l) {
            dA = std::max(dA, c->sigmaA[l]);
            dE = std::max(dE, c->sigmaE[l]);
        }

    FwdLaunch L{};
    L.m = c->view();
    L.sigmaA = c->sigA.p;
    L.sigmaE = c->sigE.p;
    L.nL = nL;
    L.seed = fw->rngSeed;
    L.B = B;
    L.score = c->score.p;
    L.visits = c->visits.p;
    L.dropped = c->dropped.p;
    L.next = c->next.p;

    FinLaunch F{};
    F.score = c->score.p;
    F.lumped = c->lumped.p;
    F.vol = c->dvol.p;
    F.beta = c->beta.p;
    F.cell = c->cell.p;
    F.dropped = c->dropped.p;
    F.visits = c->visits.p;
    F.crossings = c->crossings.p;
    F.phi = c->phi.p;
    F.rse = c->rse.p;
    F.dndt = c->dndt.p;
    F.unconverged = c->unconverged.p;
    F.C = C;
    F.Np = Np;
    F.B = B;
    F.Btot = c->Btot;
    F.nTot = c->nTot;
    F.tau = c->tau;
    F.threshold = fw->relativeStandardErrorThreshold;
    F.dndtA = dA;
    F.dndtE = dE;

    res->raysTraced = 0;
    res->crossings = 0;
    res->rayMilliseconds = 0.0;
    res->totalMilliseconds = 0.0;
    res->launches = 0;
    res->unconvergedCells = 0;
    res->kernelLaunches = 0;
    res->tallyMode = smem ? 2u : 1u;
    res->srmStatus = srm ? kSrmConverged : kSrmDisabled;
    res->srmPasses = 0;
    res->srmRemainingFraction = 0.0;
    res->srmMaxIterations = srm ? srmMaxIt : 0u;
    res->srmDivergenceStreak = srm ? srmStreak : 0u;
    res->reflectingFaces = nF;
    bool chainRan = false;

    cudaEvent_t t0 = nullptr, t1 = nullptr;
    HASE_CUDA(cudaEventCreate(&t0));
    if (cudaEventCreate(&t1) != cudaSuccess) {
        cudaEventDestroy(t0);
        return fail(HASE_CUDA_ERROR, "event creation failed");
    }
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } guard{t0, t1};
    HASE_CUDA(cudaEventRecord(t0, c->stream));

    uint64_t total = 0;
    uint32_t unconverged = 0;
    for (uint32_t launch = 0;; ++launch) {
        const uint32_t target = forwardTarget(minRays, maxRays, adaptive ? fw->adaptiveSteps : 0u, launch);
        const uint32_t M = uint32_t(target - total);
        uint32_t maxNb = 0;
        for (uint32_t b = 0; b < B; ++b) {
            const Philox4 o = philox4x32_10(b, launch, 0u, kTagFwdBatch, fw->rngSeed, kFwdKeyHi);
            L.shift[b] = double(o.x) / 4294967296.0;
            L.phase[b] = o.y;  // the batch's 32-bit offset of the wavelength sequence
            L.nb[b] = b < M ? (M - b + B - 1) / B : 0u;
            F.raysInBatch[b] += double(L.nb[b]);
            maxNb = std::max(maxNb, L.nb[b]);
        }
        L.launch = launch;
        if (c->Btot > 0.0 && M > 0) {
            // enough blocks to fill the device, no more than the rays of a batch need
            uint32_t perBatch = std::max(1u, resident / B);
            perBatch = std::min(perBatch, std::max(1u, (maxNb + block - 1) / block));
            L.blocksPerBatch = perBatch;
            HASE_CUDA(cudaMemsetAsync(c->next.p, 0, B * sizeof(uint32_t), c->stream));
            HASE_CUDA(cudaEventRecord(c->ev[0], c->stream));
            const uint32_t grid = perBatch * B;
            const size_t shm = smem ? histBytes : 0;
            if (!srm || nF == 0) {
                if (smem) fwdRayKernel<true, 0><<<grid, block, shm, c->stream>>>(L);
                else fwdRayKernel<false, 0><<<grid, block, shm, c->stream>>>(L);
                HASE_CUDA(cudaGetLastError());
                res->kernelLaunches += 1;
            } else {
                // surface-reservoir chain: the source pass deposits into
                // reservoir 0, reflected pass p reads reservoir (p - 1) % 2 and
                // deposits into p % 2; every pass is queued, batches whose
                // chain ended skip the rest on the device (no host sync)
                const size_t faces = size_t(B) * nF;
                SrmLaunch& S = L.srm;
                S.faces = c->bfaces.p;
                S.nF = nF;
                S.S = srmSlots;
                S.cdf = c->cdf.p;
                S.chain = c->chain.p;
                for (uint32_t pass = 0; pass <= srmMaxIt; ++pass) {
                    const int out = int(pass & 1u), in = 1 - out;
                    S.pass = pass;
                    S.outCounts = c->resCounts[out].p;
                    S.outFaceW = c->resW[out].p;
                    S.outSlot = c->resSlot[out].p;
                    S.outLam = c->resLam[out].p;
                    S.outRay = c->resRay[out].p;
                    S.inCounts = c->resCounts[in].p;
                    S.inSlot = c->resSlot[in].p;
                    S.inLam = c->resLam[in].p;
                    HASE_CUDA(cudaMemsetAsync(S.outCounts, 0, faces * sizeof(uint32_t), c->stream));
                    HASE_CUDA(cudaMemsetAsync(S.outFaceW, 0, faces * sizeof(double), c->stream));
                    if (pass > 0) {
                        HASE_CUDA(cudaMemsetAsync(c->next.p, 0, B * sizeof(uint32_t), c->stream));
                        for (uint32_t b = 0; b < B; ++b) {
                            const Philox4 o = philox4x32_10(b, launch, pass, kTagFwdBatch, fw->rngSeed, kFwdKeyHi);
                            L.shift[b] = double(o.x) / 4294967296.0;
                        }
                        if (smem) fwdRayKernel<true, 2><<<grid, block, shm, c->stream>>>(L);
                        else fwdRayKernel<false, 2><<<grid, block, shm, c->stream>>>(L);
                    } else {
                        if (smem) fwdRayKernel<true, 1><<<grid, block, shm, c->stream>>>(L);
                        else fwdRayKernel<false, 1><<<grid, block, shm, c->stream>>>(L);
                    }
                    HASE_CUDA(cudaGetLastError());
                    srmSortKernel<<<uint32_t((faces + 255) / 256), 256, 0, c->stream>>>(
                        S.outCounts, S.outSlot, S.outLam, S.outRay, srmSlots, faces);
                    srmScanKernel<<<B, kScanBlock, 0, c->stream>>>(S.outFaceW, c->cdf.p, nF);
                    srmControlKernel<<<1, kMaxBatches, 0, c->stream>>>(c->chain.p, c->cdf.p, nF, B, pass, srmTol,
                                                                      srmStreak);
                    HASE_CUDA(cudaGetLastError());
                    res->kernelLaunches += 4;
                }
                chainRan = true;
            }
            HASE_CUDA(cudaEventRecord(c->ev[1], c->stream));
        }
        total = target;
        F.totalRays = double(total);
        HASE_CUDA(cudaMemsetAsync(c->unconverged.p, 0, sizeof(uint32_t), c->stream));
        HASE_CUDA(cudaMemsetAsync(c->crossings.p, 0, sizeof(unsigned long long), c->stream));
        fwdFinalizeKernel<<<(C + 255) / 256, 256, 0, c->stream>>>(F);
        HASE_CUDA(cudaGetLastError());
        res->kernelLaunches += 1;
        HASE_CUDA(cudaMemcpyAsync(&unconverged, c->unconverged.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
        HASE_CUDA(cudaStreamSynchronize(c->stream));
        if (c->Btot > 0.0 && M > 0) {
            float ms = 0.0f;
            HASE_CUDA(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
            res->rayMilliseconds += ms;
        }
        res->launches = launch + 1;
        if (chainRan) {  // the last launch's chains are the ones reported
            std::vector<SrmChain> ch(B);
            HASE_CUDA(cudaMemcpy(ch.data(), c->chain.p, B * sizeof(SrmChain), cudaMemcpyDeviceToHost));
            auto priority = [](uint32_t st) {
                return st == kSrmDiverged ? 4 : st == kSrmMaxIterations ? 3 : st == kSrmStable ? 2
                                            : st == kSrmConverged ? 1 : 0;
            };
            res->srmStatus = kSrmDisabled;
            res->srmPasses = 0;
            res->srmRemainingFraction = 0.0;
            for (const SrmChain& x : ch) {
                if (priority(x.status) > priority(res->srmStatus)) res->srmStatus = x.status;
                res->srmPasses = std::max(res->srmPasses, x.passes);
                res->srmRemainingFraction = std::max(res->srmRemainingFraction, x.remaining);
            }
            chainRan = false;
        }
        if (target >= maxRays || !adaptive || unconverged == 0) break;
    }
    HASE_CUDA(cudaEventRecord(t1, c->stream));
    unsigned long long cross = 0;
    HASE_CUDA(cudaMemcpyAsync(&cross, c->crossings.p, sizeof(cross), cudaMemcpyDeviceToHost, c->stream));
    if (res->phiAse) HASE_CUDA(cudaMemcpyAsync(res->phiAse, c->phi.p, C * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    if (res->relativeStandardError)
        HASE_CUDA(cudaMemcpyAsync(res->relativeStandardError, c->rse.p, C * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (res->dndtAse) HASE_CUDA(cudaMemcpyAsync(res->dndtAse, c->dndt.p, C * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (res->totalRays) HASE_CUDA(cudaMemcpyAsync(res->totalRays, c->visits.p, C * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    std::vector<uint32_t> drop(C);
    HASE_CUDA(cudaMemcpyAsync(drop.data(), c->dropped.p, C * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    HASE_CUDA(cudaStreamSynchronize(c->stream));
    float totalMs = 0.0f;
    HASE_CUDA(cudaEventElapsedTime(&totalMs, t0, t1));
    res->totalMilliseconds = totalMs;
    res->crossings = cross;
    res->raysTraced = total;
    res->unconvergedCells = unconverged;
    uint64_t droppedTotal = 0;
    for (uint32_t k = 0; k < C; ++k) droppedTotal += drop[k];
    if (res->droppedRays) std::copy(drop.begin(), drop.end(), res->droppedRays);
    if (droppedTotal) return fail(HASE_DROPPED_RAYS, "%llu rays could not be walked", (unsigned long long)droppedTotal);
    if (unconverged) return fail(HASE_NOT_CONVERGED, "%u cells above the threshold at maxRays", unconverged);
    return HASE_OK;
}
