// hase_device.cuh -- device-side building blocks of the phi-ASE hot path:
// Philox4x32-10, the packed prism-mesh view, and the FP32 prism walk.
//
// The walk follows the legacy HASEonGPU backward method (rays from a start
// point in a prism to the sample point, crossing triangle edges through the
// neighbour table and z levels), here parametrised by the remaining distance s
// to the (image) sample point, p(s) = S + s*u, walked from s = |start - S|
// down to 0.  The exits of a prism are the largest crossing parameters below
// s: edges (2-D lines n.x = c whose outward normal points against the motion)
// and the level planes z = k*h, all relative to the sample so that the last
// prism (the one touching the sample point) ends the walk at s = 0 exactly.
// Gain anchor: g = N_tot (beta (sigmaE + sigmaA) - sigmaA), cladding
// g = -claddingAbsorption (include/kernels/forward/rayWalk.hpp:170-182).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace hase {

constexpr uint32_t kTagRay = 0u;
constexpr uint32_t kTagMap = 1u;
constexpr uint32_t kTagFar = 2u;  // far rays of the local proposal: Philox counter word 3
constexpr uint32_t kWeylStep = 0x9E3779B9u;  // 2^32 / golden ratio: the rays' wavelength sequence step
constexpr int kMaxSteps = 10000;  // bounded walk (include/kernels/forward/policyRay.hpp:386)

// ---------------------------------------------------------------- Philox ----
// Philox4x32-10, Salmon, Moraes, Dror, Shaw, "Parallel Random Numbers: As Easy
// as 1, 2, 3", SC'11: 10 rounds of two 32x32->64 multiplies with a Weyl key
// schedule.
struct Philox4 {
    uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                          uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        if (round > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
#ifdef __CUDA_ARCH__
        const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
#else
        const uint64_t p0 = uint64_t(0xD2511F53u) * c0, p1 = uint64_t(0xCD9E8D57u) * c2;
        const uint32_t hi0 = uint32_t(p0 >> 32), lo0 = uint32_t(p0);
        const uint32_t hi1 = uint32_t(p1 >> 32), lo1 = uint32_t(p1);
#endif
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
    }
    return Philox4{c0, c1, c2, c3};
}

// 24-bit uniform in (0,1): (k + 1/2) 2^-24, exact in FP32.
__device__ __forceinline__ float unit24(uint32_t k24) { return (float(k24) + 0.5f) * (1.0f / 16777216.0f); }

// ------------------------------------------------------------ mesh view ----
// Packed per-triangle walk record, 3 x float4 = 48 B:
//   r0 = (nx0, ny0, c0, nx1), r1 = (ny1, c1, nx2, ny2), r2 = (c2, nb0, nb1, nb2)
// with nb_e = (neighbour << 2 | entry edge in the neighbour) as int bits, -1 at
// the mesh boundary.  Start-point record, 2 x float4 = 32 B:
//   g0 = (ax, ay, bx-ax, by-ay), g1 = (cx-ax, cy-ay, area, 0); centroid separate.
struct MeshView {
    const float4* tri;       // [T][3]
    const float4* walk;      // [T][3]: tri with NaN normals on mesh-boundary edges (the walks' records)
    const float4* geo;       // [T][2]
    const int4* verts;       // [T] point ids of the triangle's vertices (w unused)
    const float2* centroid;  // [T]
    const float* gainBeta;   // [P] beta, NaN in cladding prisms (walk)
    const float* gTab;       // [P] g of each prism for the solve's averaged (A, B) (a monochromatic solve: its pair)
    const float* srcBeta;    // [P] beta (source weight)
    const float2* points;    // [Np]
    const float* reflect;    // [T][2] or nullptr
    // importance walks: per sample level, the slices x layers lines of a
    // triangle ordered by their layer distance to the image level (without,
    // with reflections), so that lines with similar numbers of level planes
    // share a lane slot of the line teams
    const uint16_t* lineOrder[2];
    uint32_t T, layers, P, Np;
    uint32_t divTm, divTs;   // floor(p / T) = (p * divTm) >> divTs for p < 2^31 (invariantDivisor)
    uint32_t divNpm, divNps; // the same for division by Np
    float h;                 // level spacing
    float cladAbs;           // claddingAbsorption
    float tolEnd;            // |s| below which the target is reached
    float tirCos2[2];        // total internal reflection when uz^2 <= tirCos2[surface]
};

// Layer of prism index p < 2^31 (p = t + layer T): an exact multiply-shift
// instead of a 32-bit division by the runtime T.
__device__ __forceinline__ uint32_t prismLayer(const MeshView& m, uint32_t p) {
    return uint32_t((uint64_t(p) * m.divTm) >> m.divTs);
}

// Level of sample index s < 2^31 (s = point + level Np), by multiply-shift.
__device__ __forceinline__ uint32_t sampleLevel(const MeshView& m, uint32_t s) {
    return uint32_t((uint64_t(s) * m.divNpm) >> m.divNps);
}

// Unfolded integer level of the image of sample level ls for reflection slice.
__device__ __forceinline__ int imageLevel(int ls, int layers, uint32_t slice) {
    switch (slice) {
        case 1: return -ls;                 // bottom
        case 2: return 2 * layers - ls;     // top
        case 3: return ls - 2 * layers;     // bottom, then top
        case 4: return ls + 2 * layers;     // top, then bottom
        default: return ls;
    }
}

__device__ __forceinline__ int expectedReflections(uint32_t slice) { return slice == 0 ? 0 : (slice <= 2 ? 1 : 2); }

// Legacy reflectivity index t*2 + surface (include/core/mesh.hpp:301-332), with
// total internal reflection above the critical angle.
__device__ __forceinline__ float reflectFactor(const MeshView& m, uint32_t t, int surf, float uz) {
    if (uz * uz <= m.tirCos2[surf]) return 1.0f;
    return m.reflect ? __ldg(m.reflect + 2 * t + surf) : 0.0f;
}

// One ray in flight.  The walk runs in the unfolded z coordinate (reflection
// images); `row` is the prism-index offset (physical layer x T) of the current
// unfolded layer and `rstep` the offset of the next physical layer toward the
// image point, +T or -T (it flips at every reflection), so no division, modulo
// or multiplication is needed per crossing.
struct Ray {
    uint32_t t;     // triangle
    int row;        // physical layer of the current unfolded layer, times T
    int rstep;      // +T / -T
    int reflLeft;   // reflections the slice still implies
    int steps;
    float s;        // remaining distance to the image point
    float G;        // accumulated ln(gain) for the pair (A, B), including reflection factors
    float A, B;     // g = beta*A - B: the walk's reference pair
    float Jb;       // integral of beta dl over gain prisms (beta walks)
    float Lc;       // path length in cladding prisms (kWalkBeta)
    float D;        // path length, start to image point
    float ux, uy, uz;
    // the current layer's exit plane lies at s = zl hOverUz: zl is the plane's
    // unfolded level offset from the image point (a small integer, exact in
    // float) and hOverUz = h / uz, both times the layer step toward the image
    // (-1 when uz > 0, else +1), so that zl grows by 1 per plane
    float hOverUz;
    float zl;
};

enum StepResult { kContinue = 0, kDone = 1, kDropped = 2 };

// How a walk obtains the gain coefficient g of the current prism.  The beta
// walks also keep the path integrals that make the gain of every wavelength
// (A_l, B_l) follow from the reference pair's: ln G_l = G + (A_l - A) Jb -
// (B_l - B)(D - Lc), so a ray's gain is known for the whole spectrum
// (rayMeanGain); for the reference pair it is G itself, bit for bit as the
// table walk gives it.
enum WalkMode {
    kWalkBeta = 0,         // beta from m.gainBeta; cladding prisms (NaN beta) add to Lc
    kWalkTable = 1,        // g from m.gTab (a monochromatic solve: the table is built for its pair)
    kWalkBetaNoClad = 2,   // as kWalkBeta for a medium without cladding prisms (beta is never NaN)
};

// Initialise a ray from the start point, given as its offset (dx, dy, dz)
// from the image point (Sx, Sy, kImg*h), in physical layer `layer`.
// Returns |start - image|^2.
__device__ __forceinline__ float initRay(Ray& r, uint32_t t, int layer, float dx, float dy, float dz, int kImg,
                                         uint32_t slice, float A, float B, const MeshView& m) {
    const float h = m.h;
    if (dz == 0.0f) dz = 1e-6f * h;  // a ray inside a level plane: nudge it off the plane
    const float D2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    const float D = sqrtf(D2);
    const float inv = 1.0f / D;
    r.t = t;
    r.row = layer * int(m.T);
    r.reflLeft = expectedReflections(slice);
    r.steps = 0;
    r.s = D;
    r.G = 0.0f;
    r.Jb = 0.0f;
    r.Lc = 0.0f;
    r.D = D;
    r.ux = dx * inv;
    r.uy = dy * inv;
    r.uz = dz * inv;
    // moving toward the image: down (layer step -1) when uz > 0, up (+1) otherwise
    const float hu = __fdividef(h, r.uz);
    r.hOverUz = r.uz > 0.0f ? -hu : hu;
    r.zl = r.uz > 0.0f ? float(kImg - layer) : float(layer + 1 - kImg);
    r.rstep = r.uz > 0.0f ? -int(m.T) : int(m.T);
    r.A = A;
    r.B = B;
    return D2;
}

// One segment of length len in a prism whose table value (kWalkTable: g) or
// beta (NaN: cladding) is gb.
template <int WALK>
__device__ __forceinline__ void addSegment(Ray& r, float gb, float len, float cladAbs) {
    if constexpr (WALK == kWalkTable) {
        r.G = fmaf(gb, len, r.G);
    } else if constexpr (WALK == kWalkBetaNoClad) {
        r.G = fmaf(fmaf(gb, r.A, -r.B), len, r.G);
        r.Jb = fmaf(gb, len, r.Jb);
    } else {
        const bool gain = gb == gb;
        r.G = fmaf(gain ? fmaf(gb, r.A, -r.B) : -cladAbs, len, r.G);
        r.Jb = fmaf(gain ? gb : 0.0f, len, r.Jb);
        r.Lc += gain ? 0.0f : len;
    }
}

// ln gain of a finished ray (beta walks) for the pair (A_l, B_l): exact for
// the reference pair.
__device__ __forceinline__ float rayLnGain(const Ray& r, float Al, float Bl) {
    return fmaf(Al - r.A, r.Jb, fmaf(r.B - Bl, r.D - r.Lc, r.G));
}

// The mean over the nL wavelengths (A_l, B_l) of a finished ray's gain
// (beta walks), relative to the reference pair's exact exp(G) (FP64 above
// G = 80): one FP32 exponential per wavelength of the difference of its
// exponent from G, (A_l - A) Jb - (B_l - B)(D - Lc) (bounded by the spread
// of the cross sections along one path; clamped at 80).  One wavelength:
// exp(G), as the table walk.
__device__ __forceinline__ double rayMeanGain(const Ray& r, const float2* spec, uint32_t nL) {
    const double e = r.G < 80.0f ? double(expf(r.G)) : exp(double(r.G));
    if (nL == 1) return e;
    const float Lg = r.D - r.Lc;
    float sum = 0.0f;
    for (uint32_t l = 0; l < nL; ++l) {
        const float2 ab = __ldg(spec + l);
        sum += __expf(fminf(fmaf(ab.x - r.A, r.Jb, (r.B - ab.y) * Lg), 80.0f));
    }
    return e * double(sum) / double(nL);
}

// One triangle column: the edge exit of the current triangle (edge exits are
// compared as fractions num/den by cross multiplication; one approximate
// division gives the chosen exit parameter), then every level plane crossed
// before it.
// Walks up to K triangle columns per call.  Once a column's exit edge is
// known, the next triangle's walk record is loaded (into the registers the
// current record no longer needs) while the current column's level planes are
// worked through, so its latency is hidden behind them.
// The walk is bound by instruction issue, so the level-plane loop is kept
// short: the step bound is checked once per call (the loop itself ends
// within 3 x layers crossings: every physical layer step reaches a surface and
// at most two reflections are allowed), and kWalkTable walks the table of g = beta A
// - B (m.gTab) instead of evaluating it at every crossing (WalkMode).
template <int K = 1, int WALK = kWalkBeta, typename Loader>
__device__ __forceinline__ int stepRay(const MeshView& m, float Sx, float Sy, Ray& r, Loader&& load) {
    const float* gcol = WALK == kWalkTable ? m.gTab : m.gainBeta;
    float4 a, b, c;
    load(r.t, a, b, c);
    // beta (kWalkTable: g) of the current prism, issued with the record so
    // that its latency overlaps the edge tests
    float gb = __ldg(gcol + r.row + r.t);
#pragma unroll 1
    for (int k = 0; k < K; ++k) {
        float bn = -1.0f, bd = 0.0f;  // best fraction so far (-1/0 = -inf)
        int bw = -1;
        const auto edge = [&](float nx, float ny, float cc, int nbw) {
            const float dd = -fmaf(nx, r.ux, ny * r.uy);       // > 0: moving out through the edge
            const float nm = fmaf(nx, Sx, fmaf(ny, Sy, -cc));  // signed distance of the sample from the edge line
            // Boundary edges are never exits: the 2-D mesh is convex and the
            // target lies in it, so only rounding could route a ray across one.
            // The walk records (MeshView::walk) give them NaN normals, so
            // their dd > 0 test fails.  The entry edge needs no test either:
            // the two triangles of an edge store exactly negated normals (both
            // are computed in FP64 from the same two points and rounded), so
            // the entry edge's dd is exactly minus the dd > 0 it was chosen
            // with in the previous triangle.
            const bool ok = dd > 0.0f;
            if (ok && nm * bd > bn * dd) {
                bn = nm;
                bd = dd;
                bw = nbw;
            }
        };
        edge(a.x, a.y, a.z, __float_as_int(c.y));
        edge(a.w, b.x, b.y, __float_as_int(c.z));
        edge(b.z, b.w, c.x, __float_as_int(c.w));
        // clamped at 0: the comparison sz < sEdge below is reached only with
        // sz > tolEnd >= 0, where the clamp does not change it
        const float sEdge = fmaxf(fminf(__fdividef(bn, bd), r.s), 0.0f);
        if (K > 1 && k + 1 < K && bw >= 0) load(uint32_t(bw) >> 2, a, b, c);
        // Level planes crossed before the edge exit: the triangle, and with it
        // sEdge, stays the same, so they cost no edge test.
        while (true) {
            const float sz = fminf(r.zl * r.hOverUz, r.s);
            const float next = fmaxf(sEdge, sz);
            if (next <= m.tolEnd) {
                addSegment<WALK>(r, gb, r.s, m.cladAbs);
                r.s = 0.0f;
                return kDone;
            }
            addSegment<WALK>(r, gb, r.s - next, m.cladAbs);
            r.s = next;
            ++r.steps;
            if (sz < sEdge) break;
            const int cand = r.row + r.rstep;
            if (uint32_t(cand) >= m.P) {  // a physical bottom/top surface: reflect
                if (r.reflLeft <= 0) return kDropped;
                r.G += __logf(reflectFactor(m, r.t, cand < 0 ? 0 : 1, r.uz));
                --r.reflLeft;
                r.rstep = -r.rstep;
            } else {
                r.row = cand;
            }
            r.zl += 1.0f;
            gb = __ldg(gcol + r.row + r.t);
        }
        r.t = uint32_t(bw) >> 2;
        if (K > 1 && k + 1 < K) gb = __ldg(gcol + r.row + r.t);
    }
    // the step bound, once per call: a call walks at most K columns of at most
    // 1 + 3 x layers segments each
    return r.steps >= kMaxSteps ? kDropped : kContinue;
}

// After kDone: a reflection the slice implies but which happens at the target
// itself (a sample on the reflecting surface) is applied in the final triangle.
__device__ __forceinline__ void finishReflections(const MeshView& m, Ray& r) {
    if (r.reflLeft > 0) {
        r.G += __logf(reflectFactor(m, r.t, r.row + r.rstep < 0 ? 0 : 1, r.uz));
        r.reflLeft = 0;
    }
}

// Near-field start point for a prism (t, l) that touches the image point of
// sample point `pS` (a vertex of triangle t at image level kImg = l or l+1).
// Uniform start points give such prisms an infinite-variance 1/d^2 weight;
// here the direction from the image point is uniform in the prism's solid
// angle (azimuth uniform between the two triangle edges at the vertex,
// sin(elevation) uniform: the prism seen from its vertex is that lune
// segment, solid angle alpha) and the distance is uniform up to the prism
// exit L(Omega).  The density is 1/(alpha L d^2), so the ray weight
// beta G / d^2 / density = beta G alpha L stays bounded.
// Returns false when t does not have pS as a vertex.
__device__ __forceinline__ bool nearFieldStart(const MeshView& m, uint32_t t, int l, int kImg, uint32_t pS,
                                               float2 S, float uAz, float uEl, float uR, float& dx, float& dy,
                                               float& dz, float& alphaL) {
    const int4 v = __ldg(m.verts + t);
    const int iv = v.x == int(pS) ? 0 : (v.y == int(pS) ? 1 : (v.z == int(pS) ? 2 : -1));
    if (iv < 0) return false;
    const float4 g0 = __ldg(m.geo + 2 * t), g1 = __ldg(m.geo + 2 * t + 1);
    const float px[3] = {g0.x, g0.x + g0.z, g0.x + g1.x};
    const float py[3] = {g0.y, g0.y + g0.w, g0.y + g1.y};
    float e1x = (iv == 0 ? px[1] : (iv == 1 ? px[2] : px[0])) - S.x;
    float e1y = (iv == 0 ? py[1] : (iv == 1 ? py[2] : py[0])) - S.y;
    float e2x = (iv == 0 ? px[2] : (iv == 1 ? px[0] : px[1])) - S.x;
    float e2y = (iv == 0 ? py[2] : (iv == 1 ? py[0] : py[1])) - S.y;
    const float i1 = rsqrtf(e1x * e1x + e1y * e1y), i2 = rsqrtf(e2x * e2x + e2y * e2y);
    e1x *= i1;
    e1y *= i1;
    e2x *= i2;
    e2y *= i2;
    const float cosA = fminf(fmaxf(fmaf(e1x, e2x, e1y * e2y), -1.0f), 1.0f);
    const float alpha = acosf(cosA);
    const float sinA = sinf(alpha);
    // slerp weights: sin(u a)/sin a and sin((1-u) a)/sin a = cos(u a) - cos a sin(u a)/sin a
    float su, cu;
    sincosf(uAz * alpha, &su, &cu);
    const float w2 = __fdividef(su, sinA), w1 = fmaf(-cosA, w2, cu);
    const float cx = fmaf(w1, e1x, w2 * e2x), cy = fmaf(w1, e1y, w2 * e2y);
    const float se = uEl, ce = sqrtf(fmaxf(0.0f, 1.0f - se * se));
    // edge opposite the vertex: edge (iv + 1) % 3 of the walk record
    const int eo = iv == 2 ? 0 : iv + 1;
    const float4 r0 = __ldg(m.tri + 3 * t), r1 = __ldg(m.tri + 3 * t + 1), r2 = __ldg(m.tri + 3 * t + 2);
    const float nx = eo == 0 ? r0.x : (eo == 1 ? r0.w : r1.z);
    const float ny = eo == 0 ? r0.y : (eo == 1 ? r1.x : r1.w);
    const float cc = eo == 0 ? r0.z : (eo == 1 ? r1.y : r2.x);
    const float lxy = __fdividef(cc - fmaf(nx, S.x, ny * S.y), fmaf(nx, cx, ny * cy));
    const float L = fminf(__fdividef(lxy, ce), __fdividef(m.h, se));
    const float r = uR * L;
    const float zs = l == kImg ? 1.0f : -1.0f;
    dx = r * ce * cx;
    dy = r * ce * cy;
    dz = zs * r * se;
    alphaL = alpha * L;
    return true;
}

struct GlobalLoader {
    const float4* tri;
    __device__ __forceinline__ void operator()(uint32_t t, float4& a, float4& b, float4& c) const {
        a = __ldg(tri + 3 * t);
        b = __ldg(tri + 3 * t + 1);
        c = __ldg(tri + 3 * t + 2);
    }
};

}  // namespace hase
