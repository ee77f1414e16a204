// hase_oracle.cpp -- FP64 CPU restatement of the backward prism phi-ASE method.
//
// TEST INFRASTRUCTURE ONLY (the checker): the product library never links
// this file.  See hase_oracle.h for the reference anchors this follows.
//
// Method (Eckert et al., CPC 207 (2016) 362; legacy HASEonGPU v1 layout):
//   phi(s) = N_tot / (4 pi tau) * Int_V beta(x) G(x->s) / |s-x|^2 dV,
//   G(x->s) = exp(Int g dl) * (reflection factors),  g = N_tot (beta (sE+sA) - sA)
//   (cladding prisms: g = -claddingAbsorption).
// Estimator: prism p (of reflection slice j) is drawn with probability q_jp/Q
// from the straight-line importance weight w_jp = beta_p V_p G(c_p->s_j)/|s_j-c_p|^2
// (c_p the prism centre, s_j the image of s for slice j), the start point is
// uniform in the prism, and each ray contributes
//   X = N_tot/(4 pi tau) * beta_p V_p (Q/q_jp) G / d^2.
// Rays are assigned to prisms by systematic sampling of the integer CDF of q
// (one Philox phase per sample and pass), so the ray->prism map is integer and
// reproducible bit for bit.  phi = sum X / N, mse = sqrt(|<X^2>-<X>^2|/N)/<X>
// (the legacy relative error), adaptive passes top up samples whose mse is
// above the threshold to the geometric ray target of include/core/types.hpp:333-354.
#include "hase_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <utility>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr uint32_t kPhiloxM0 = 0xD2511F53u;
constexpr uint32_t kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u;
constexpr uint32_t kPhiloxW1 = 0xBB67AE85u;
constexpr uint32_t kTagRay = 0u;
constexpr uint32_t kTagMap = 1u;
constexpr int kMaxSteps = 10000;
constexpr double kPi = 3.14159265358979323846;

void philox(const uint32_t in[4], const uint32_t k[2], uint32_t out[4]) {
    uint32_t c0 = in[0], c1 = in[1], c2 = in[2], c3 = in[3];
    uint32_t k0 = k[0], k1 = k[1];
    for (int round = 0; round < 10; ++round) {
        if (round > 0) {
            k0 += kPhiloxW0;
            k1 += kPhiloxW1;
        }
        const uint64_t p0 = uint64_t(kPhiloxM0) * c0;
        const uint64_t p1 = uint64_t(kPhiloxM1) * c2;
        const uint32_t n0 = uint32_t(p1 >> 32) ^ c1 ^ k0;
        const uint32_t n1 = uint32_t(p1);
        const uint32_t n2 = uint32_t(p0 >> 32) ^ c3 ^ k1;
        const uint32_t n3 = uint32_t(p0);
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// 24-bit uniform in (0,1): (k + 0.5) * 2^-24, exact in FP32 and FP64.
inline double unit(uint32_t x) { return (double(x >> 8) + 0.5) * (1.0 / 16777216.0); }

struct Tables {
    uint32_t T = 0;
    std::vector<int32_t> nbr, forb;
    std::vector<double> nx, ny, c, cx, cy, area;
};

int buildTables(uint32_t np, const double* pts, uint32_t T, const uint32_t* tri, Tables& t) {
    t.T = T;
    t.nbr.assign(3 * T, -1);
    t.forb.assign(3 * T, -1);
    t.nx.resize(3 * T); t.ny.resize(3 * T); t.c.resize(3 * T);
    t.cx.resize(T); t.cy.resize(T); t.area.resize(T);
    std::map<std::pair<uint32_t, uint32_t>, std::pair<uint32_t, int>> open;
    for (uint32_t i = 0; i < T; ++i) {
        const uint32_t v[3] = {tri[3 * i], tri[3 * i + 1], tri[3 * i + 2]};
        for (int e = 0; e < 3; ++e)
            if (v[e] >= np) return -1;
        const double x0 = pts[2 * v[0]], y0 = pts[2 * v[0] + 1];
        const double x1 = pts[2 * v[1]], y1 = pts[2 * v[1] + 1];
        const double x2 = pts[2 * v[2]], y2 = pts[2 * v[2] + 1];
        const double cross = (x1 - x0) * (y2 - y0) - (y1 - y0) * (x2 - x0);
        if (cross == 0.0) return -2;
        const double orient = cross > 0 ? 1.0 : -1.0;
        t.cx[i] = (x0 + x1 + x2) / 3.0;
        t.cy[i] = (y0 + y1 + y2) / 3.0;
        t.area[i] = 0.5 * std::fabs(cross);
        for (int e = 0; e < 3; ++e) {
            const uint32_t a = v[e], b = v[(e + 1) % 3];
            const double ex = pts[2 * b] - pts[2 * a], ey = pts[2 * b + 1] - pts[2 * a + 1];
            const double inv = 1.0 / std::sqrt(ex * ex + ey * ey);
            // (ey, -ex) is the right-hand normal of a->b: outward for CCW triangles.
            const double nx = orient * ey * inv, ny = -orient * ex * inv;
            t.nx[3 * i + e] = nx;
            t.ny[3 * i + e] = ny;
            t.c[3 * i + e] = nx * pts[2 * a] + ny * pts[2 * a + 1];
            const auto key = std::make_pair(std::min(a, b), std::max(a, b));
            auto it = open.find(key);
            if (it == open.end()) {
                open.emplace(key, std::make_pair(i, e));
            } else {
                const uint32_t j = it->second.first;
                const int f = it->second.second;
                if (t.nbr[3 * j + f] != -1) return -3;  // non-manifold edge
                t.nbr[3 * i + e] = int32_t(j);
                t.forb[3 * i + e] = f;
                t.nbr[3 * j + f] = int32_t(i);
                t.forb[3 * j + f] = e;
                open.erase(it);
            }
        }
    }
    return 0;
}

struct Model {
    const oracle_mesh* m;
    Tables tab;
    uint32_t T, L, layers, P, Np;
    double h, H, extent;
    std::vector<double> gainA, gainB;  // per wavelength: g = beta*A - B
    double meanA = 0, meanB = 0;
};

int makeModel(const oracle_mesh* m, const oracle_spectrum* sp, Model& md) {
    md.m = m;
    if (m->numberOfLevels < 2 || m->numberOfTriangles == 0 || sp->numberOfWavelengths == 0) return -1;
    int rc = buildTables(m->numberOfPoints, m->points, m->numberOfTriangles, m->triangles, md.tab);
    if (rc) return rc;
    md.T = m->numberOfTriangles;
    md.L = m->numberOfLevels;
    md.layers = md.L - 1;
    md.P = md.T * md.layers;
    md.Np = m->numberOfPoints;
    md.h = m->thickness;
    md.H = md.h * md.layers;
    double ext = md.H;
    for (uint32_t i = 0; i < md.Np; ++i)
        ext = std::max(ext, std::max(std::fabs(m->points[2 * i]), std::fabs(m->points[2 * i + 1])));
    md.extent = ext;
    for (uint32_t l = 0; l < sp->numberOfWavelengths; ++l) {
        md.gainA.push_back(m->nTot * (sp->sigmaE[l] + sp->sigmaA[l]));
        md.gainB.push_back(m->nTot * sp->sigmaA[l]);
    }
    for (uint32_t l = 0; l < sp->numberOfWavelengths; ++l) {
        md.meanA += md.gainA[l] / sp->numberOfWavelengths;
        md.meanB += md.gainB[l] / sp->numberOfWavelengths;
    }
    return 0;
}

inline bool isCladding(const Model& md, uint32_t t) {
    return md.m->claddingCellTypes && md.m->claddingCellTypes[t] == md.m->claddingNumber;
}

inline double gainCoeff(const Model& md, uint32_t t, uint32_t layer, double A, double B) {
    if (isCladding(md, t)) return -md.m->claddingAbsorption;
    return md.m->betaVolume[size_t(layer) * md.T + t] * A - B;
}

// Unfolded z of the image of a sample at height zs for reflection slice j.
inline double imageZ(double zs, double H, uint32_t slice) {
    switch (slice) {
        case 1: return -zs;            // bottom
        case 2: return 2.0 * H - zs;   // top
        case 3: return zs - 2.0 * H;   // bottom, then top
        case 4: return zs + 2.0 * H;   // top, then bottom
        default: return zs;
    }
}

inline int floorDiv(int a, int b) { int q = a / b; if ((a % b != 0) && ((a < 0) != (b < 0))) --q; return q; }
inline int floorMod(int a, int b) { return a - floorDiv(a, b) * b; }

inline uint32_t physicalLayer(int lu, uint32_t layers) {
    const int m = floorMod(lu, int(2 * layers));
    return m < int(layers) ? uint32_t(m) : uint32_t(2 * layers - 1 - m);
}

// Reflection factor at physical surface `surf` (0 bottom, 1 top) of triangle t
// for a ray with |cos(incidence)| = cz: total internal reflection above the
// critical angle, otherwise the legacy per-triangle reflectivity t*2 + surf.
inline double reflectFactor(const Model& md, uint32_t t, int surf, double cz) {
    const double* n = md.m->refractiveIndices;
    const double nin = n ? n[2 * surf] : 1.0, nout = n ? n[2 * surf + 1] : 1.0;
    if (nout < nin) {
        const double sinI = std::sqrt(std::max(0.0, 1.0 - cz * cz));
        if (sinI >= nout / nin) return 1.0;
    }
    return md.m->reflectivities ? md.m->reflectivities[2 * t + surf] : 0.0;
}

struct Walk {
    double lnGain;  // for the (A, B) passed to walk
    double dist;
    bool dropped;
    // path integrals every wavelength's ln gain is linear in:
    // ln G_l = A_l jb - B_l lg - claddingAbsorption lc + lnR
    double jb, lg, lc, lnR;
};

// Walk from start (x0,y0,z0) in prism (t, level) to the (image) target.
Walk walk(const Model& md, double x0, double y0, double z0, uint32_t t, uint32_t level, double Sx,
          double Sy, double Sz, uint32_t slice, double A, double B) {
    const Tables& tb = md.tab;
    double ux = x0 - Sx, uy = y0 - Sy, uz = z0 - Sz;
    const double D = std::sqrt(ux * ux + uy * uy + uz * uz);
    Walk w{0.0, D, false, 0.0, 0.0, 0.0, 0.0};
    if (D == 0.0) return w;
    ux /= D; uy /= D; uz /= D;
    const double tol = 1e-9 * md.extent;
    int lu = int(level);
    int forbidden = -1;
    double s = D, G = 0.0, lnR = 0.0;
    int reflections = 0;
    const int expected = slice == 0 ? 0 : (slice <= 2 ? 1 : 2);
    for (int step = 0;; ++step) {
        if (step >= kMaxSteps) { w.dropped = true; break; }
        double best = -std::numeric_limits<double>::infinity();
        int bestEdge = -1;
        for (int e = 0; e < 3; ++e) {
            if (e == forbidden) continue;
            const double den = tb.nx[3 * t + e] * ux + tb.ny[3 * t + e] * uy;
            if (!(den < 0.0)) continue;
            if (tb.nbr[3 * t + e] < 0) continue;  // convex mesh: boundary edges are never exits
            double se = (tb.nx[3 * t + e] * Sx + tb.ny[3 * t + e] * Sy - tb.c[3 * t + e]) / (-den);
            if (se > s) se = s;
            if (se > best) { best = se; bestEdge = e; }
        }
        double sz = -std::numeric_limits<double>::infinity();
        int dl = 0;
        if (uz > 0.0) { sz = (double(lu) * md.h - Sz) / uz; dl = -1; }
        else if (uz < 0.0) { sz = (double(lu + 1) * md.h - Sz) / uz; dl = +1; }
        if (sz > s) sz = s;
        const uint32_t phys = physicalLayer(lu, md.layers);
        const double g = gainCoeff(md, t, phys, A, B);
        const bool clad = isCladding(md, t);
        const double beta = clad ? 0.0 : md.m->betaVolume[size_t(phys) * md.T + t];
        const double next = std::max(std::max(best, sz), 0.0);
        const double len = next <= tol ? s : s - next;
        G += g * len;
        if (clad) w.lc += len;
        else { w.jb += beta * len; w.lg += len; }
        if (next <= tol) {  // the target lies in (or on the boundary of) this prism
            s = 0.0;
            break;
        }
        s = next;
        if (sz >= best) {
            // level plane k = lu (down) or lu + 1 (up)
            const int k = dl < 0 ? lu : lu + 1;
            if (floorMod(k, int(md.layers)) == 0) {
                const int surf = floorMod(floorDiv(k, int(md.layers)), 2);  // 0 bottom, 1 top
                if (reflections >= expected) { w.dropped = true; break; }
                const double R = reflectFactor(md, t, surf, std::fabs(uz));
                lnR += R > 0.0 ? std::log(R) : -std::numeric_limits<double>::infinity();
                ++reflections;
            }
            lu += dl;
        } else {
            const int32_t n = tb.nbr[3 * t + bestEdge];
            forbidden = tb.forb[3 * t + bestEdge];
            t = uint32_t(n);
        }
    }
    if (!w.dropped && reflections < expected) {
        // The target itself lies on the reflecting surface: the remaining
        // bounce happens at the target, in the final triangle.
        const int k = int(std::lround(Sz / md.h));
        const int surf = floorMod(floorDiv(k, int(md.layers)), 2);
        const double R = reflectFactor(md, t, surf, std::fabs(uz));
        lnR += R > 0.0 ? std::log(R) : -std::numeric_limits<double>::infinity();
    }
    w.lnGain = G + lnR;
    w.lnR = lnR;
    return w;
}

uint64_t rayMap(uint32_t n, const float* w, uint32_t rays, uint32_t phase, uint32_t* q, uint32_t* off) {
    float wmax = 0.0f;
    for (uint32_t i = 0; i < n; ++i) wmax = std::max(wmax, w[i]);
    uint64_t Q = 0;
    if (wmax > 0.0f) {
        const double scale = 16777216.0 / double(wmax);
        for (uint32_t i = 0; i < n; ++i) {
            q[i] = w[i] > 0.0f ? uint32_t(std::ceil(double(w[i]) * scale)) : 0u;
            Q += q[i];
        }
    } else {
        for (uint32_t i = 0; i < n; ++i) q[i] = 0;
    }
    if (Q == 0) {
        for (uint32_t i = 0; i <= n; ++i) off[i] = 0;
        return 0;
    }
    using u128 = unsigned __int128;
    const u128 den = u128(Q) << 32;
    uint64_t C = 0;
    for (uint32_t b = 0; b <= n; ++b) {
        const u128 num = (u128(C) * rays << 32) + u128(phase) * Q;
        off[b] = uint32_t(num / den);
        if (b < n) C += q[b];
    }
    return Q;
}

uint32_t adaptiveTarget(const oracle_experiment* e, uint32_t k) {
    if (e->maxRays <= e->minRays || e->adaptiveSteps == 0) return e->minRays;
    if (k >= e->adaptiveSteps) return e->maxRays;
    const double growth = std::pow(double(e->maxRays) / double(e->minRays), 1.0 / double(e->adaptiveSteps));
    const double target = double(e->minRays) * std::pow(growth, double(k));
    const uint32_t r = uint32_t(std::ceil(target));
    return std::min(std::max(r, e->minRays), e->maxRays);
}

void samplePoint(const Model& md, uint32_t sample, double& x, double& y, double& z) {
    const uint32_t p = sample % md.Np, l = sample / md.Np;
    x = md.m->points[2 * p];
    y = md.m->points[2 * p + 1];
    z = double(l) * md.h;
}

void importance(const Model& md, uint32_t sample, uint32_t slices, double* w) {
    double Sx, Sy, Sz;
    samplePoint(md, sample, Sx, Sy, Sz);
    for (uint32_t j = 0; j < slices; ++j) {
        const double Iz = imageZ(Sz, md.H, j);
        for (uint32_t l = 0; l < md.layers; ++l)
            for (uint32_t t = 0; t < md.T; ++t) {
                const size_t p = size_t(l) * md.T + t;
                const double beta = md.m->betaVolume[p];
                double& out = w[size_t(j) * md.P + p];
                if (!(beta > 0.0)) { out = 0.0; continue; }
                const double z0 = (double(l) + 0.5) * md.h;
                const Walk r = walk(md, md.tab.cx[t], md.tab.cy[t], z0, t, l, Sx, Sy, Iz, j, md.meanA, md.meanB);
                if (r.dropped || r.dist == 0.0) { out = 0.0; continue; }
                out = beta * md.tab.area[t] * md.h * std::exp(r.lnGain) / (r.dist * r.dist);
            }
    }
}

}  // namespace

extern "C" {

void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) { philox(ctr, key, out); }

int oracle_build_tables(uint32_t np, const double* pts, uint32_t T, const uint32_t* tri, int32_t* nbr,
                        int32_t* forb, double* nx, double* ny, double* c, double* cx, double* cy, double* area) {
    Tables t;
    const int rc = buildTables(np, pts, T, tri, t);
    if (rc) return rc;
    std::memcpy(nbr, t.nbr.data(), 3 * T * sizeof(int32_t));
    std::memcpy(forb, t.forb.data(), 3 * T * sizeof(int32_t));
    std::memcpy(nx, t.nx.data(), 3 * T * sizeof(double));
    std::memcpy(ny, t.ny.data(), 3 * T * sizeof(double));
    std::memcpy(c, t.c.data(), 3 * T * sizeof(double));
    std::memcpy(cx, t.cx.data(), T * sizeof(double));
    std::memcpy(cy, t.cy.data(), T * sizeof(double));
    std::memcpy(area, t.area.data(), T * sizeof(double));
    return 0;
}

int oracle_trace(const oracle_mesh* mesh, const oracle_spectrum* spectrum, uint32_t wavelength, uint32_t n,
                 const double* start, const uint32_t* tri, const uint32_t* level, const uint32_t* sample,
                 const uint32_t* slice, double* lnGain, double* distance, uint32_t* dropped) {
    Model md;
    const int rc = makeModel(mesh, spectrum, md);
    if (rc) return rc;
    if (wavelength >= spectrum->numberOfWavelengths) return -1;
    for (uint32_t i = 0; i < n; ++i) {
        double Sx, Sy, Sz;
        samplePoint(md, sample[i], Sx, Sy, Sz);
        const Walk r = walk(md, start[3 * i], start[3 * i + 1], start[3 * i + 2], tri[i], level[i], Sx, Sy,
                            imageZ(Sz, md.H, slice[i]), slice[i], md.gainA[wavelength], md.gainB[wavelength]);
        lnGain[i] = r.lnGain;
        distance[i] = r.dist;
        dropped[i] = r.dropped ? 1u : 0u;
    }
    return 0;
}

int oracle_importance(const oracle_mesh* mesh, const oracle_spectrum* spectrum, uint32_t sample, uint32_t slices,
                      double* weights) {
    Model md;
    const int rc = makeModel(mesh, spectrum, md);
    if (rc) return rc;
    importance(md, sample, slices, weights);
    return 0;
}

uint64_t oracle_ray_map(uint32_t n, const float* weights, uint32_t rays, uint32_t phase, uint32_t* q,
                        uint32_t* offsets) {
    return rayMap(n, weights, rays, phase, q, offsets);
}

int oracle_phi_ase(const oracle_mesh* mesh, const oracle_spectrum* spectrum, const oracle_experiment* ex,
                   const float* weightsOverride, int threads, oracle_result* res) {
    Model md;
    int rc = makeModel(mesh, spectrum, md);
    if (rc) return rc;
    if (ex->maxSample < ex->minSample || ex->maxSample >= md.Np * md.L || ex->minRays == 0) return -10;
    const uint32_t slices = ex->useReflections ? 5u : 1u;
    const uint32_t nW = slices * md.P;
    const uint32_t nS = ex->maxSample - ex->minSample + 1;
    const uint32_t nLambda = spectrum->numberOfWavelengths;
    const double C = mesh->nTot / (4.0 * kPi * mesh->crystalTFluo);
    const uint32_t key[2] = {ex->seed, 0u};
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
#pragma omp parallel
    {
        std::vector<double> wd(nW);
        std::vector<float> wf(nW);
        std::vector<uint32_t> q(nW), off(nW + 1);
#pragma omp for schedule(dynamic, 1)
        for (uint32_t i = 0; i < nS; ++i) {
            const uint32_t s = ex->minSample + i;
            if (weightsOverride) {
                std::memcpy(wf.data(), weightsOverride + size_t(i) * nW, nW * sizeof(float));
            } else {
                importance(md, s, slices, wd.data());
                for (uint32_t k = 0; k < nW; ++k) wf[k] = float(wd[k]);
            }
            double Sx, Sy, Sz;
            samplePoint(md, s, Sx, Sy, Sz);
            double sum = 0.0, sum2 = 0.0;
            uint32_t total = 0, dropped = 0;
            double mse = 0.0;
            for (uint32_t pass = 0;; ++pass) {
                const uint32_t target = adaptiveTarget(ex, pass);
                if (target > total) {
                    const uint32_t M = target - total;
                    uint32_t pc[4] = {0u, s, pass, kTagMap}, po[4];
                    philox(pc, key, po);
                    const uint64_t Q = rayMap(nW, wf.data(), M, po[0], q.data(), off.data());
                    if (Q == 0) { total = target; break; }
                    for (uint32_t r = 0; r < M; ++r) {
                        const uint32_t b = uint32_t(std::upper_bound(off.begin(), off.end(), r) - off.begin()) - 1u;
                        const uint32_t j = b / md.P, p = b % md.P;
                        const uint32_t t = p % md.T, l = p / md.T;
                        uint32_t rc4[4] = {r, s, pass, kTagRay}, ro[4];
                        philox(rc4, key, ro);
                        const uint32_t* v = mesh->triangles + 3 * t;
                        const double Iz = imageZ(Sz, md.H, j);
                        const int kImg = int(std::lround(Iz / md.h));
                        const uint32_t pS = s % md.Np;
                        const int iv = v[0] == pS ? 0 : (v[1] == pS ? 1 : (v[2] == pS ? 2 : -1));
                        double x, y, z, factor;  // factor: the start density's volume term
                        if (ex->nearField && (int(l) == kImg || int(l) + 1 == kImg) && iv >= 0) {
                            // solid angle of the prism at the (image) sample point: see nearFieldStart
                            const uint32_t va = v[(iv + 1) % 3], vb = v[(iv + 2) % 3];
                            double e1x = mesh->points[2 * va] - Sx, e1y = mesh->points[2 * va + 1] - Sy;
                            double e2x = mesh->points[2 * vb] - Sx, e2y = mesh->points[2 * vb + 1] - Sy;
                            const double i1 = 1.0 / std::sqrt(e1x * e1x + e1y * e1y), i2 = 1.0 / std::sqrt(e2x * e2x + e2y * e2y);
                            e1x *= i1; e1y *= i1; e2x *= i2; e2y *= i2;
                            const double alpha = std::acos(std::min(1.0, std::max(-1.0, e1x * e2x + e1y * e2y)));
                            const double uAz = unit(ro[0]), se = unit(ro[2]), uR = unit(ro[3]);
                            const double w1 = std::sin((1.0 - uAz) * alpha) / std::sin(alpha);
                            const double w2 = std::sin(uAz * alpha) / std::sin(alpha);
                            const double cx = w1 * e1x + w2 * e2x, cy = w1 * e1y + w2 * e2y;
                            const double ce = std::sqrt(std::max(0.0, 1.0 - se * se));
                            const int eo = (iv + 1) % 3;
                            const double nx = md.tab.nx[3 * t + eo], ny = md.tab.ny[3 * t + eo], cc = md.tab.c[3 * t + eo];
                            const double lxy = (cc - (nx * Sx + ny * Sy)) / (nx * cx + ny * cy);
                            const double L = std::min(lxy / ce, md.h / se);
                            const double rr = uR * L;
                            const double zs = int(l) == kImg ? 1.0 : -1.0;
                            x = Sx + rr * ce * cx;
                            y = Sy + rr * ce * cy;
                            z = double(kImg) * md.h + zs * rr * se;
                            factor = alpha * L;  // start density 1/(alpha L d^2)
                        } else {
                            uint32_t k1 = ro[0] >> 8, k2 = ro[1] >> 8;
                            if (uint64_t(k1) + k2 + 1u > (1u << 24)) { k1 = (1u << 24) - 1u - k1; k2 = (1u << 24) - 1u - k2; }
                            const double u1 = (double(k1) + 0.5) / 16777216.0, u2 = (double(k2) + 0.5) / 16777216.0;
                            const double ax = mesh->points[2 * v[0]], ay = mesh->points[2 * v[0] + 1];
                            x = ax + u1 * (mesh->points[2 * v[1]] - ax) + u2 * (mesh->points[2 * v[2]] - ax);
                            y = ay + u1 * (mesh->points[2 * v[1] + 1] - ay) + u2 * (mesh->points[2 * v[2] + 1] - ay);
                            z = (double(l) + unit(ro[2])) * md.h;
                            factor = -1.0;  // uniform in the prism: density 1/V
                        }
                        const Walk wk = walk(md, x, y, z, t, l, Sx, Sy, Iz, j, md.meanA, md.meanB);
                        if (wk.dropped || wk.dist == 0.0) { ++dropped; continue; }
                        const double vol = factor > 0.0 ? factor : md.tab.area[t] * md.h / (wk.dist * wk.dist);
                        // the ray's gain averaged over the spectrum (no wavelength is drawn)
                        double eg = 0.0;
                        for (uint32_t lam = 0; lam < nLambda; ++lam)
                            eg += std::exp(md.gainA[lam] * wk.jb - md.gainB[lam] * wk.lg -
                                           mesh->claddingAbsorption * wk.lc + wk.lnR);
                        eg /= double(nLambda);
                        const double X = C * mesh->betaVolume[p] * vol * (double(Q) / double(q[b])) * eg;
                        sum += X;
                        sum2 += X * X;
                    }
                    total = target;
                }
                const double mean = sum / total;
                mse = mean > 0.0 ? std::sqrt(std::fabs(sum2 / total - mean * mean) / total) / mean : 0.0;
                if (mse <= ex->mseThreshold || target >= ex->maxRays || pass >= ex->adaptiveSteps) break;
            }
            const double phi = sum / total;
            res->phiAse[i] = phi;
            res->mse[i] = mse;
            res->totalRays[i] = total;
            res->droppedRays[i] = dropped;
            if (res->gainSum) res->gainSum[i] = sum;
            if (res->gainSumSquare) res->gainSumSquare[i] = sum2;
            if (res->dndtAse) {
                double sA = 0, sE = 0;
                for (uint32_t l = 0; l < nLambda; ++l) { sA = std::max(sA, spectrum->sigmaA[l]); sE = std::max(sE, spectrum->sigmaE[l]); }
                if (nLambda == 1) { sA = spectrum->sigmaA[0]; sE = spectrum->sigmaE[0]; }
                const double bc = mesh->betaCells ? mesh->betaCells[s] : 0.0;
                res->dndtAse[i] = (bc * (sE + sA) - sA) * double(float(phi));
            }
        }
    }
    return 0;
}

}  // extern "C"
