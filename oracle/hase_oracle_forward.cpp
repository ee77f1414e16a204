// hase_oracle_forward.cpp -- FP64 CPU restatement of HASEonGPU's forward
// Tet4 phi-ASE estimator (the reference's current calcPhiASE).
//
// TEST INFRASTRUCTURE ONLY (the checker): the product library never links
// this file.  Method (reference paths):
//   source rays   include/kernels/forward/accumulation.hpp:369-453,
//                 include/kernels/forward/volumeSampling.hpp:19-161
//                 (stratified beta*V CDF per statistical batch, uniform point
//                 in the tet from four exponentials paired with the corners
//                 in ascending point index, isotropic direction; the
//                 wavelength bin from a golden-ratio sequence over the
//                 batch's rays, this build's choice: the reference draws
//                 it per ray)
//   walk + tally  include/kernels/forward/rayWalk.hpp:106-208,
//                 include/kernels/forward/accumulation.hpp:300-352
//                 (barycentric face planes; per crossed cell the tally
//                 weight * G * (exp(g l) - 1)/g split to the four material
//                 vertices by the segment-midpoint barycentric weights,
//                 then G *= exp(g l); rays escape at the mesh boundary)
//   finalise      include/kernels/forwardPhiAseMapping.hpp:51-150,
//                 include/kernels/vertexAccumulation.hpp:17-68
//                 (vertex -> cell density through lumped material vertex
//                 volumes, estimate S B / (N V) * N_tot/tau, relative error
//                 of the batch means, cells with dropped rays never converge)
//   adaptive loop include/core/forwardPhiAseEvaluator.hpp:114-178 (rays of a
//                 launch are added to the previous launches).
// The random streams are this project's own Philox4x32-10 counters (the
// reference's alpaka generator layout is not pinned bit for bit).
#include "hase_oracle.h"

#include <algorithm>
#include <numeric>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr uint32_t kTagFwdBatch = 2u;
constexpr uint32_t kTagFwdRay = 3u;
constexpr uint32_t kFwdKeyHi = 1u;
constexpr int kMaxSteps = 10000;
constexpr double kPi = 3.14159265358979323846;

inline double unit(uint32_t x) { return (double(x >> 8) + 0.5) * (1.0 / 16777216.0); }

struct TetTables {
    uint32_t C = 0, Np = 0;
    std::vector<int32_t> nbr, nbrFace;  // [C][4]
    std::vector<double> grad;           // [C][4][3]
    std::vector<double> plane;          // [C][4][4]: lambda_f(x) = a.x + d
    std::vector<double> vol;            // [C]
};

int buildTetTables(const oracle_tet_mesh* m, TetTables& t) {
    t.C = m->numberOfCells;
    t.Np = m->numberOfPoints;
    t.nbr.assign(4 * size_t(t.C), -1);
    t.nbrFace.assign(4 * size_t(t.C), -1);
    t.grad.assign(12 * size_t(t.C), 0.0);
    t.plane.assign(16 * size_t(t.C), 0.0);
    t.vol.assign(t.C, 0.0);
    std::map<std::tuple<uint32_t, uint32_t, uint32_t>, std::pair<uint32_t, int>> open;
    for (uint32_t c = 0; c < t.C; ++c) {
        const uint32_t* v = m->cells + 4 * size_t(c);
        for (int k = 0; k < 4; ++k)
            if (v[k] >= t.Np) return -1;
        const double* p0 = m->points + 3 * size_t(v[0]);
        double E[3][3];  // columns e_k = v_k - v0
        for (int k = 1; k < 4; ++k)
            for (int d = 0; d < 3; ++d) E[d][k - 1] = m->points[3 * size_t(v[k]) + d] - p0[d];
        const double det = E[0][0] * (E[1][1] * E[2][2] - E[1][2] * E[2][1]) -
                           E[0][1] * (E[1][0] * E[2][2] - E[1][2] * E[2][0]) +
                           E[0][2] * (E[1][0] * E[2][1] - E[1][1] * E[2][0]);
        if (!(std::fabs(det) > 0.0)) return -2;
        t.vol[c] = std::fabs(det) / 6.0;
        // rows of E^-1 are the gradients of lambda_1..3
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
        double* g = &t.grad[12 * size_t(c)];
        for (int d = 0; d < 3; ++d) {
            g[3 + d] = inv[0][d];
            g[6 + d] = inv[1][d];
            g[9 + d] = inv[2][d];
            g[d] = -(inv[0][d] + inv[1][d] + inv[2][d]);
        }
        // plane form (include/core/mesh.hpp:657-727): d_f = delta_f0 - grad_f . v0
        double* pl = &t.plane[16 * size_t(c)];
        for (int f = 0; f < 4; ++f) {
            pl[4 * f] = g[3 * f];
            pl[4 * f + 1] = g[3 * f + 1];
            pl[4 * f + 2] = g[3 * f + 2];
            pl[4 * f + 3] = (f == 0 ? 1.0 : 0.0) - (g[3 * f] * p0[0] + g[3 * f + 1] * p0[1] + g[3 * f + 2] * p0[2]);
        }
        // face f is opposite vertex f
        for (int f = 0; f < 4; ++f) {
            uint32_t a[3], n = 0;
            for (int k = 0; k < 4; ++k)
                if (k != f) a[n++] = v[k];
            std::sort(a, a + 3);
            const auto key = std::make_tuple(a[0], a[1], a[2]);
            auto it = open.find(key);
            if (it == open.end()) {
                open.emplace(key, std::make_pair(c, f));
            } else {
                const uint32_t o = it->second.first;
                const int of = it->second.second;
                if (t.nbr[4 * o + of] != -1) return -3;  // face shared by more than two cells
                t.nbr[4 * c + f] = int32_t(o);
                t.nbrFace[4 * c + f] = of;
                t.nbr[4 * o + of] = int32_t(c);
                t.nbrFace[4 * o + of] = f;
                open.erase(it);
            }
        }
    }
    return 0;
}

struct FwdModel {
    const oracle_tet_mesh* m;
    TetTables tab;
    std::vector<double> prefix;  // inclusive beta*V prefix
    double Btot = 0.0;
    std::vector<uint32_t> matVertex;  // [C][4]
    std::vector<double> lumped;       // [2 Np]
};

inline bool isClad(const oracle_tet_mesh* m, uint32_t c) {
    return m->claddingCellTypes && m->claddingCellTypes[c] == m->claddingNumber;
}

inline double gainCoeff(const oracle_tet_mesh* m, uint32_t c, double sA, double sE) {
    if (isClad(m, c)) return -m->claddingAbsorption;
    return m->nTot * (m->betaVolume[c] * (sE + sA) - sA);
}

// Walk one source ray from x in cell c along unit direction u.  With score
// != NULL, adds the tally of every crossed cell to score[c*4 + k] (vertex k of
// cell c) and counts the visit in visits[c]; with path != NULL, records every
// segment (cell, length, g l).  Returns -1 when the ray escaped through the
// mesh boundary, else the cell in which the walk failed.
//
// Exit face: among the faces whose coordinate decreases along u (the entry
// face excluded), the one reached first, length max(-lambda/dlambda, 0); the
// lowest face index wins a tie.  A ray through an edge or a vertex therefore
// takes zero-length steps through the cells around it until it is in a cell
// that it enters with positive length.
struct Segment {
    uint32_t cell;
    double length, gl;
};

// G0: the ray's starting weight (1 for a source ray, the reservoir's source
// weight for a reflected ray); ff0: its entry face (-1: none).  On escape,
// exitCell / exitFace / Gout (when given) receive the boundary face and the
// weight times the accumulated gain at it.
int64_t walkForward(const FwdModel& md, uint32_t c, double x[3], const double u[3], double sA, double sE,
                    double* score, uint32_t* visits, std::vector<Segment>* path, double G0 = 1.0, int ff0 = -1,
                    uint32_t* exitCell = nullptr, int* exitFace = nullptr, double* Gout = nullptr) {
    const oracle_tet_mesh* m = md.m;
    int ff = ff0;
    double G = G0;
    for (int step = 0; step < kMaxSteps; ++step) {
        const double* pl = &md.tab.plane[16 * size_t(c)];
        double lam[4], dl[4];
        double best = DBL_MAX;
        int bf = -1;
        for (int f = 0; f < 4; ++f) {
            lam[f] = pl[4 * f] * x[0] + pl[4 * f + 1] * x[1] + pl[4 * f + 2] * x[2] + pl[4 * f + 3];
            dl[f] = pl[4 * f] * u[0] + pl[4 * f + 1] * u[1] + pl[4 * f + 2] * u[2];
            if (f == ff || !(dl[f] < 0.0)) continue;
            const double len = std::max(-lam[f] / dl[f], 0.0);
            if (len < best) {
                best = len;
                bf = f;
            }
        }
        if (bf < 0) return int64_t(c);
        const double gc = gainCoeff(m, c, sA, sE);
        const double gl = gc * best;
        if (path) path->push_back(Segment{c, best, gl});
        if (score) {
            const double T = std::fabs(gl) < 1e-8 ? best : std::expm1(gl) / gc;
            const double contribution = G * T;
            if (!std::isfinite(contribution)) return int64_t(c);
            double w[4], wsum = 0.0;
            for (int f = 0; f < 4; ++f) {
                w[f] = std::max(0.0, lam[f] + 0.5 * best * dl[f]);
                wsum += w[f];
            }
            for (int f = 0; f < 4; ++f)
                score[4 * size_t(c) + f] += contribution * (wsum > DBL_EPSILON ? w[f] / wsum : 0.25);
            ++visits[c];
            G *= std::exp(gl);
        }
        for (int d = 0; d < 3; ++d) x[d] += u[d] * best;
        const int32_t n = md.tab.nbr[4 * size_t(c) + bf];
        if (n < 0) {  // escaped through the boundary
            if (exitCell) *exitCell = c;
            if (exitFace) *exitFace = bf;
            if (Gout) *Gout = G;
            return -1;
        }
        ff = md.tab.nbrFace[4 * size_t(c) + bf];
        c = uint32_t(n);
    }
    return int64_t(c);
}

}  // namespace

namespace {

void philoxFwd(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t seed, uint32_t out[4]) {
    const uint32_t ctr[4] = {c0, c1, c2, c3}, key[2] = {seed, kFwdKeyHi};
    oracle_philox4x32_10(ctr, key, out);
}

uint32_t fwdTarget(const oracle_forward_experiment* e, uint32_t k) {
    if (e->maxRays <= e->minRays || e->adaptiveSteps == 0) return e->minRays;
    if (k >= e->adaptiveSteps) return e->maxRays;
    const double growth = std::pow(double(e->maxRays) / double(e->minRays), 1.0 / double(e->adaptiveSteps));
    const uint32_t r = uint32_t(std::ceil(double(e->minRays) * std::pow(growth, double(k))));
    return std::min(std::max(r, e->minRays), e->maxRays);
}

// ---- surface-reservoir reflections (include/core/forwardSrm.hpp:100-365,
// include/kernels/forward/accumulation.hpp:455-833) ----

// A boundary face with a reflecting surface (surface id > 0): outward unit
// normal normalize((b - a) x (c - a)) turned away from the cell centre
// (include/kernels/forward/rayWalk.hpp:60-84), centroid (the reflected rays'
// start point, rayWalk.hpp:44-58), reflectivity and squared index ratio
// n_inside / n_outside (-1: no total internal reflection) as
// include/core/mesh.hpp:301-332 resolve them.
struct BFace {
    uint32_t c;
    int f;
    double n[3], cen[3], R, ratio2;
};

void buildBoundaryFaces(const FwdModel& md, std::vector<BFace>& faces) {
    const oracle_tet_mesh* m = md.m;
    faces.clear();
    if (!m->cellFaceBoundaries) return;
    for (uint32_t c = 0; c < m->numberOfCells; ++c) {
        const uint32_t* v = m->cells + 4 * size_t(c);
        for (int f = 0; f < 4; ++f) {
            const int32_t id = m->cellFaceBoundaries[4 * size_t(c) + f];
            if (md.tab.nbr[4 * size_t(c) + f] >= 0 || id <= 0) continue;
            BFace b{};
            b.c = c;
            b.f = f;
            const double* P[3];
            int n = 0;
            for (int k = 0; k < 4; ++k)
                if (k != f) P[n++] = m->points + 3 * size_t(v[k]);
            double e1[3], e2[3], cc[3] = {0, 0, 0}, cen[3] = {0, 0, 0};
            for (int d = 0; d < 3; ++d) {
                e1[d] = P[1][d] - P[0][d];
                e2[d] = P[2][d] - P[0][d];
                b.cen[d] = (P[0][d] + P[1][d] + P[2][d]) / 3.0;
                for (int k = 0; k < 4; ++k) cc[d] += m->points[3 * size_t(v[k]) + d] / 4.0;
                cen[d] = b.cen[d];
            }
            double nn[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
            const double len = std::sqrt(nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2]);
            for (int d = 0; d < 3; ++d) nn[d] /= len;
            if (nn[0] * (cc[0] - cen[0]) + nn[1] * (cc[1] - cen[1]) + nn[2] * (cc[2] - cen[2]) > 0.0)
                for (int d = 0; d < 3; ++d) nn[d] = -nn[d];
            for (int d = 0; d < 3; ++d) b.n[d] = nn[d];
            const uint32_t sid = uint32_t(id);
            if (m->surfaceReflectivities && sid < m->numberOfSurfaces) b.R = m->surfaceReflectivities[sid];
            else b.R = m->reflectivities ? m->reflectivities[2 * size_t(c) + f % 2] : 0.0;
            double nIn, nOut;
            if (m->surfaceRefractiveIndexInside && sid < m->numberOfSurfaces) nIn = m->surfaceRefractiveIndexInside[sid];
            else nIn = m->refractiveIndices ? m->refractiveIndices[2 * (f % 2)] : 1.0;
            if (m->surfaceRefractiveIndexOutside && sid < m->numberOfSurfaces)
                nOut = m->surfaceRefractiveIndexOutside[sid];
            else nOut = m->refractiveIndices ? m->refractiveIndices[2 * (f % 2) + 1] : 1.0;
            b.ratio2 = (nIn > 0.0 && nOut > 0.0) ? (nIn / nOut) * (nIn / nOut) : -1.0;
            faces.push_back(b);
        }
    }
}

// include/kernels/reflection.hpp:21-47
double boundaryReflectance(const BFace& b, const double u[3]) {
    const double un = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    const double cosI = std::min(1.0, std::fabs((u[0] * b.n[0] + u[1] * b.n[1] + u[2] * b.n[2]) / un));
    const double sin2 = std::max(0.0, 1.0 - cosI * cosI);
    if (b.ratio2 > 0.0 && b.ratio2 * sin2 > 1.0) return 1.0;
    return std::max(0.0, b.R);
}

struct Reservoir {
    uint32_t S = 0, nF = 0, B = 0;
    std::vector<uint32_t> counts, lam;     // [B][nF], [B][nF][S]
    std::vector<double> faceW, dir, w;     // [B][nF], [B][nF][S][3], [B][nF][S]
    void init(uint32_t b, uint32_t f, uint32_t s) {
        B = b;
        nF = f;
        S = s;
        counts.assign(size_t(B) * nF, 0u);
        faceW.assign(size_t(B) * nF, 0.0);
        lam.assign(size_t(B) * nF * S, 0u);
        w.assign(size_t(B) * nF * S, 0.0);
        dir.assign(size_t(B) * nF * S * 3, 0.0);
    }
    void clear() {
        std::fill(counts.begin(), counts.end(), 0u);
        std::fill(faceW.begin(), faceW.end(), 0.0);
    }
};

// A ray that left the mesh through reflecting face k of batch b.
struct Deposit {
    uint32_t ray, b, k, lam;
    double G, u[3];
};

// include/kernels/forward/accumulation.hpp:455-506: weighted reservoir of
// reflected directions per face; uA, uB decide a replacement once the face's
// slots are full.
void deposit(Reservoir& res, const BFace& bf, const Deposit& d, double uA, double uB) {
    if (res.S == 0 || !(d.G > 0.0) || !std::isfinite(d.G)) return;
    const double w = d.G * boundaryReflectance(bf, d.u);
    if (!(w > 0.0) || !std::isfinite(w)) return;
    const size_t face = size_t(d.b) * res.nF + d.k;
    const uint32_t seen = res.counts[face]++;
    const double prior = res.faceW[face];
    res.faceW[face] += w;
    uint32_t slot = seen;
    if (slot >= res.S) {
        const double p = std::min(1.0, double(res.S) * w / (prior + w));
        if (uA >= p) return;
        slot = std::min(res.S - 1, uint32_t(uB * double(res.S)));
    }
    const double dn = d.u[0] * bf.n[0] + d.u[1] * bf.n[1] + d.u[2] * bf.n[2];
    double r[3];
    for (int k = 0; k < 3; ++k) r[k] = d.u[k] - bf.n[k] * (2.0 * dn);
    const double rl = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    const size_t s = face * res.S + slot;
    for (int k = 0; k < 3; ++k) res.dir[3 * s + k] = rl > DBL_EPSILON ? r[k] / rl : 0.0;
    res.w[s] = w;
    res.lam[s] = d.lam;
}

// Status of one batch's reflection chain (include/core/forwardSrm.hpp:281-363).
struct SrmChain {
    double initial = 0.0, prev = 0.0, remaining = 0.0;
    uint32_t grow = 0, status = 0, passes = 0;
    bool active = false;
};

enum : uint32_t { kSrmDisabled = 0, kSrmConverged = 1, kSrmStable = 2, kSrmDiverged = 3, kSrmMaxIterations = 4 };

uint32_t srmPriority(uint32_t s) {
    switch (s) {
        case kSrmDisabled: return 0;
        case kSrmConverged: return 1;
        case kSrmStable: return 2;
        case kSrmMaxIterations: return 3;
        default: return 4;
    }
}

}  // namespace

extern "C" {

int oracle_tet_tables(const oracle_tet_mesh* mesh, int32_t* neighbors, int32_t* neighborFace, double* gradients,
                      double* volumes) {
    TetTables t;
    const int rc = buildTetTables(mesh, t);
    if (rc) return rc;
    std::memcpy(neighbors, t.nbr.data(), t.nbr.size() * sizeof(int32_t));
    std::memcpy(neighborFace, t.nbrFace.data(), t.nbrFace.size() * sizeof(int32_t));
    std::memcpy(gradients, t.grad.data(), t.grad.size() * sizeof(double));
    std::memcpy(volumes, t.vol.data(), t.vol.size() * sizeof(double));
    return 0;
}

int oracle_forward_phi_ase(const oracle_tet_mesh* m, const oracle_spectrum* sp, const oracle_forward_experiment* ex,
                           int threads, oracle_forward_result* res) {
    FwdModel md;
    md.m = m;
    int rc = buildTetTables(m, md.tab);
    if (rc) return rc;
    if (ex->minRays == 0 || ex->batches < 2 || sp->numberOfWavelengths == 0) return -10;
    const uint32_t C = m->numberOfCells, Np = m->numberOfPoints, B = ex->batches;
    const uint32_t nL = sp->numberOfWavelengths;
    md.prefix.resize(C);
    double acc = 0.0;
    for (uint32_t c = 0; c < C; ++c) {
        acc += m->betaVolume[c] * md.tab.vol[c];
        md.prefix[c] = acc;
    }
    md.Btot = acc;
    md.matVertex.resize(4 * size_t(C));
    md.lumped.assign(2 * size_t(Np), 0.0);
    for (uint32_t c = 0; c < C; ++c)
        for (int k = 0; k < 4; ++k) {
            const uint32_t mv = m->cells[4 * size_t(c) + k] + (isClad(m, c) ? Np : 0u);
            md.matVertex[4 * size_t(c) + k] = mv;
            md.lumped[mv] += md.tab.vol[c] / 4.0;
        }
    uint32_t lastSource = 0;
    for (uint32_t c = 0; c < C; ++c)
        if (m->betaVolume[c] * md.tab.vol[c] > 0.0) lastSource = c;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    std::vector<double> score(size_t(B) * 4 * C, 0.0);  // [batch][cell][vertex]
    std::vector<uint32_t> dropped(C, 0), visits(C, 0), raysInBatch(B, 0);
    // reflections: reflecting boundary faces, face index per (cell, face), two reservoirs
    const bool srm = ex->useReflections != 0;
    std::vector<BFace> bfaces;
    std::vector<int32_t> bidx;
    Reservoir resA, resB;
    if (srm) {
        buildBoundaryFaces(md, bfaces);
        bidx.assign(4 * size_t(C), -1);
        for (size_t k = 0; k < bfaces.size(); ++k) bidx[4 * size_t(bfaces[k].c) + bfaces[k].f] = int32_t(k);
        resA.init(B, uint32_t(bfaces.size()), ex->surfaceReservoirSize);
        resB.init(B, uint32_t(bfaces.size()), ex->surfaceReservoirSize);
    }
    res->srmStatus = kSrmDisabled;
    res->srmPasses = 0;
    res->srmRemainingFraction = 0.0;
    auto applyDeposits = [&](std::vector<Deposit>& deps, Reservoir& into, uint32_t launch, uint32_t pass) {
        std::sort(deps.begin(), deps.end(), [](const Deposit& a, const Deposit& b) { return a.ray < b.ray; });
        for (const Deposit& d : deps) {
            uint32_t o[4];
            philoxFwd(d.ray, launch, (pass << 2) | 2u, kTagFwdRay, ex->seed, o);
            deposit(into, bfaces[d.k], d, unit(o[0]), unit(o[1]));
        }
        deps.clear();
    };
    // The reflected passes of one launch (include/core/forwardSrm.hpp:216-363):
    // per batch, nb rays per pass drawn from the input reservoir (face by a
    // stratified target in the face-weight CDF, slot by weight), started at
    // the face centroid with the previous pass's total weight / nb, their
    // own boundary hits deposited into the other reservoir.
    auto reflectPasses = [&](uint32_t launch, const std::vector<uint32_t>& nb) {
        const uint32_t nF = uint32_t(bfaces.size()), S = resA.S;
        std::vector<SrmChain> chain(B);
        Reservoir* in = &resA;
        Reservoir* out = &resB;
        std::vector<double> cdf(size_t(B) * nF);
        auto scan = [&](const Reservoir& r) {
            std::vector<double> tot(B, 0.0);
            for (uint32_t b = 0; b < B; ++b) {
                double acc = 0.0;
                for (uint32_t k = 0; k < nF; ++k) {
                    acc += r.faceW[size_t(b) * nF + k];
                    cdf[size_t(b) * nF + k] = acc;
                }
                tot[b] = acc;
            }
            return tot;
        };
        std::vector<double> W = scan(*in);
        for (uint32_t b = 0; b < B; ++b) {
            if (W[b] == 0.0) {
                chain[b].status = kSrmConverged;
                continue;
            }
            chain[b].initial = chain[b].prev = W[b];
            chain[b].status = kSrmMaxIterations;
            chain[b].remaining = 1.0;
            chain[b].active = true;
        }
        const uint32_t M = uint32_t(std::accumulate(nb.begin(), nb.end(), uint64_t(0)));
        for (uint32_t pass = 1; pass <= ex->reflectionMaxIterations; ++pass) {
            bool any = false;
            for (uint32_t b = 0; b < B; ++b) any = any || chain[b].active;
            if (!any) break;
            out->clear();
            std::vector<double> shift(B);
            for (uint32_t b = 0; b < B; ++b) {
                uint32_t o[4];
                philoxFwd(b, launch, pass, kTagFwdBatch, ex->seed, o);
                shift[b] = double(o[0]) / 4294967296.0;
            }
            std::vector<Deposit> deps;
#pragma omp parallel
            {
                std::vector<double> local(size_t(B) * 4 * C, 0.0);
                std::vector<uint32_t> ldrop(C, 0), lvisit(C, 0);
                std::vector<Deposit> ldeps;
#pragma omp for schedule(dynamic, 4096)
                for (uint32_t r = 0; r < M; ++r) {
                    const uint32_t b = r % B, i = r / B;
                    if (!chain[b].active || S == 0 || nF == 0) continue;
                    const double* cb = &cdf[size_t(b) * nF];
                    const double t = (double(i) + shift[b]) / double(nb[b]) * cb[nF - 1];
                    uint32_t k = uint32_t(std::upper_bound(cb, cb + nF, t) - cb);
                    if (k >= nF) k = nF - 1;
                    const size_t face = size_t(b) * nF + k;
                    const uint32_t filled = std::min(in->counts[face], S);
                    if (filled == 0) continue;
                    double slotSum = 0.0;
                    for (uint32_t q = 0; q < filled; ++q) slotSum += in->w[face * S + q];
                    if (!(slotSum > 0.0)) continue;
                    uint32_t o[4];
                    philoxFwd(r, launch, pass << 2, kTagFwdRay, ex->seed, o);
                    const double target = unit(o[0]) * slotSum;
                    double cum = 0.0;
                    uint32_t slot = filled - 1;
                    for (uint32_t q = 0; q < filled; ++q) {
                        cum += in->w[face * S + q];
                        if (cum >= target) {
                            slot = q;
                            break;
                        }
                    }
                    const size_t si = face * S + slot;
                    double u[3] = {in->dir[3 * si], in->dir[3 * si + 1], in->dir[3 * si + 2]};
                    const double ul = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
                    for (int d = 0; d < 3; ++d) u[d] = ul > DBL_EPSILON ? u[d] / ul : 0.0;
                    const BFace& bf = bfaces[k];
                    double x[3] = {bf.cen[0], bf.cen[1], bf.cen[2]};
                    const uint32_t lam = in->lam[si];
                    uint32_t ec = 0;
                    int ef = -1;
                    double eg = 0.0;
                    const int64_t fail = walkForward(md, bf.c, x, u, sp->sigmaA[lam], sp->sigmaE[lam],
                                                     &local[size_t(b) * 4 * C], lvisit.data(), nullptr,
                                                     chain[b].prev / double(nb[b]), bf.f, &ec, &ef, &eg);
                    if (fail >= 0) ++ldrop[size_t(fail)];
                    else if (bidx[4 * size_t(ec) + ef] >= 0)
                        ldeps.push_back(Deposit{r, b, uint32_t(bidx[4 * size_t(ec) + ef]), lam, eg, {u[0], u[1], u[2]}});
                }
#pragma omp critical
                {
                    for (size_t k = 0; k < local.size(); ++k) score[k] += local[k];
                    for (uint32_t c = 0; c < C; ++c) {
                        dropped[c] += ldrop[c];
                        visits[c] += lvisit[c];
                    }
                    deps.insert(deps.end(), ldeps.begin(), ldeps.end());
                }
            }
            applyDeposits(deps, *out, launch, pass);
            std::swap(in, out);
            W = scan(*in);
            for (uint32_t b = 0; b < B; ++b) {
                SrmChain& ch = chain[b];
                if (!ch.active) continue;
                const double cur = W[b];
                ch.passes = pass;
                ch.remaining = cur / ch.initial;
                if (cur > ch.prev) {
                    if (++ch.grow >= ex->divergenceStreak) {
                        ch.status = kSrmDiverged;
                        ch.active = false;
                        continue;
                    }
                } else {
                    ch.grow = 0;
                    if (std::fabs(cur - ch.prev) / std::max(cur, 1.0e-30) < ex->reflectionTolerance) {
                        ch.status = kSrmStable;
                        ch.active = false;
                        continue;
                    }
                }
                if (ch.remaining < ex->reflectionTolerance) {
                    ch.status = kSrmConverged;
                    ch.active = false;
                    continue;
                }
                ch.prev = cur;
            }
        }
        res->srmStatus = kSrmDisabled;
        res->srmPasses = 0;
        res->srmRemainingFraction = 0.0;
        for (uint32_t b = 0; b < B; ++b) {
            if (srmPriority(chain[b].status) > srmPriority(res->srmStatus)) res->srmStatus = chain[b].status;
            res->srmPasses = std::max(res->srmPasses, chain[b].passes);
            res->srmRemainingFraction = std::max(res->srmRemainingFraction, chain[b].remaining);
        }
    };
    uint64_t total = 0;
    double sA = sp->sigmaA[0], sE = sp->sigmaE[0];
    for (uint32_t l = 1; l < nL; ++l) { sA = std::max(sA, sp->sigmaA[l]); sE = std::max(sE, sp->sigmaE[l]); }
    uint32_t launch = 0;
    for (;; ++launch) {
        const uint32_t target = fwdTarget(ex, launch);
        const uint32_t M = uint32_t(target - total);
        std::vector<double> shift(B);
        std::vector<uint32_t> phase(B), nb(B);
        for (uint32_t b = 0; b < B; ++b) {
            uint32_t o[4];
            philoxFwd(b, launch, 0u, kTagFwdBatch, ex->seed, o);
            shift[b] = double(o[0]) / 4294967296.0;
            phase[b] = o[1];
            nb[b] = b < M ? (M - b + B - 1) / B : 0u;
            raysInBatch[b] += nb[b];
        }
        std::vector<Deposit> deps;
        if (srm) resA.clear();
        if (md.Btot > 0.0) {
#pragma omp parallel
            {
                std::vector<double> local(size_t(B) * 4 * C, 0.0);
                std::vector<uint32_t> ldrop(C, 0), lvisit(C, 0);
                std::vector<Deposit> ldeps;
#pragma omp for schedule(dynamic, 4096)
                for (uint32_t r = 0; r < M; ++r) {
                    const uint32_t b = r % B, i = r / B;
                    const double t = (double(i) + shift[b]) / double(nb[b]) * md.Btot;
                    uint32_t c = uint32_t(std::upper_bound(md.prefix.begin(), md.prefix.end(), t) - md.prefix.begin());
                    if (c >= C) c = lastSource;
                    uint32_t o[4], o2[4];
                    philoxFwd(r, launch, 0u, kTagFwdRay, ex->seed, o);
                    philoxFwd(r, launch, 1u, kTagFwdRay, ex->seed, o2);
                    double e[4], esum = 0.0;
                    for (int k = 0; k < 4; ++k) { e[k] = -std::log(unit(o[k])); esum += e[k]; }
                    // exponential k goes to the corner of k-th smallest point index
                    uint32_t v[4];
                    for (int k = 0; k < 4; ++k) v[k] = m->cells[4 * size_t(c) + k];
                    std::sort(v, v + 4);
                    double x[3] = {0.0, 0.0, 0.0};
                    for (int k = 0; k < 4; ++k) {
                        const double* p = m->points + 3 * size_t(v[k]);
                        for (int d = 0; d < 3; ++d) x[d] += e[k] / esum * p[d];
                    }
                    const double z = 2.0 * unit(o2[0]) - 1.0, phi = 2.0 * kPi * unit(o2[1]);
                    const double rr = std::sqrt(std::max(0.0, 1.0 - z * z));
                    const double u[3] = {rr * std::cos(phi), rr * std::sin(phi), z};
                    const uint32_t lam = uint32_t((uint64_t(uint32_t(i * 0x9E3779B9u + phase[b])) * nL) >> 32);
                    uint32_t ec = 0;
                    int ef = -1;
                    double eg = 0.0;
                    const int64_t fail = walkForward(md, c, x, u, sp->sigmaA[lam], sp->sigmaE[lam],
                                                     &local[size_t(b) * 4 * C], lvisit.data(), nullptr, 1.0, -1, &ec,
                                                     &ef, &eg);
                    if (fail >= 0) ++ldrop[size_t(fail)];
                    else if (srm && bidx[4 * size_t(ec) + ef] >= 0)
                        ldeps.push_back(Deposit{r, b, uint32_t(bidx[4 * size_t(ec) + ef]), lam, eg, {u[0], u[1], u[2]}});
                }
#pragma omp critical
                {
                    for (size_t k = 0; k < local.size(); ++k) score[k] += local[k];
                    for (uint32_t c = 0; c < C; ++c) {
                        dropped[c] += ldrop[c];
                        visits[c] += lvisit[c];
                    }
                    deps.insert(deps.end(), ldeps.begin(), ldeps.end());
                }
            }
        }
        if (srm) {
            applyDeposits(deps, resA, launch, 0u);
            reflectPasses(launch, nb);
        }
        total = target;
        // finalise
        std::vector<double> vscore(size_t(B) * 2 * Np, 0.0);
        for (uint32_t b = 0; b < B; ++b)
            for (size_t k = 0; k < 4 * size_t(C); ++k)
                vscore[size_t(b) * 2 * Np + md.matVertex[k]] += score[size_t(b) * 4 * C + k];
        bool converged = true;
        for (uint32_t c = 0; c < C; ++c) {
            const double V = md.tab.vol[c];
            double sum = 0.0, mSum = 0.0, m2Sum = 0.0;
            uint32_t active = 0;
            for (uint32_t b = 0; b < B; ++b) {
                double dens = 0.0;
                for (int k = 0; k < 4; ++k) {
                    const uint32_t mv = md.matVertex[4 * size_t(c) + k];
                    dens += md.lumped[mv] > 0.0 ? vscore[size_t(b) * 2 * Np + mv] / md.lumped[mv] : 0.0;
                }
                const double bs = dens / 4.0 * V;
                sum += bs;
                if (raysInBatch[b] == 0) continue;
                const double mean = bs / double(raysInBatch[b]);
                mSum += mean;
                m2Sum += mean * mean;
                ++active;
            }
            const double estimate = sum * md.Btot / (double(total) * V);
            double rse = DBL_MAX;
            if (dropped[c] == 0 && active >= 2) {
                const double mean = mSum / active;
                if (mean == 0.0) {
                    rse = NAN;
                } else {
                    const double var = std::max(0.0, (m2Sum - mSum * mSum / active) / (active - 1.0));
                    rse = std::sqrt(var / active) / std::fabs(mean);
                }
            }
            const double phi = double(float(estimate * m->nTot / m->crystalTFluo));
            res->phiAse[c] = phi;
            res->relativeStandardError[c] = rse;
            if (res->dndtAse) {
                const double a = nL == 1 ? sp->sigmaA[0] : sA, e = nL == 1 ? sp->sigmaE[0] : sE;
                res->dndtAse[c] = (m->betaVolume[c] * (e + a) - a) * phi;
            }
            if (res->droppedRays) res->droppedRays[c] = dropped[c];
            if (res->rayVisits) res->rayVisits[c] = visits[c];
            if (!(std::isfinite(rse) && rse <= ex->rseThreshold)) converged = false;
        }
        if (target >= ex->maxRays || ex->maxRays <= ex->minRays || ex->adaptiveSteps == 0 || converged) break;
    }
    res->totalRays = total;
    res->launches = launch + 1;
    return 0;
}

int oracle_tet_trace(const oracle_tet_mesh* m, const oracle_spectrum* sp, uint32_t wavelength, uint32_t n,
                     const uint32_t* startCell, const double* origin, const double* direction, uint32_t maxSegments,
                     uint32_t* segments, uint32_t* cells, double* lengths, double* lnGain, double* endPoint,
                     int32_t* status) {
    FwdModel md;
    md.m = m;
    const int rc = buildTetTables(m, md.tab);
    if (rc) return rc;
    if (wavelength >= sp->numberOfWavelengths) return -10;
    for (uint32_t i = 0; i < n; ++i) {
        if (startCell[i] >= m->numberOfCells) return -11;
        double x[3] = {origin[3 * i], origin[3 * i + 1], origin[3 * i + 2]};
        std::vector<Segment> path;
        const int64_t fail = walkForward(md, startCell[i], x, direction + 3 * size_t(i), sp->sigmaA[wavelength],
                                         sp->sigmaE[wavelength], nullptr, nullptr, &path);
        segments[i] = uint32_t(path.size());
        double lg = 0.0;
        for (size_t k = 0; k < path.size(); ++k) {
            lg += path[k].gl;
            if (k < maxSegments) {
                if (cells) cells[size_t(i) * maxSegments + k] = path[k].cell;
                if (lengths) lengths[size_t(i) * maxSegments + k] = path[k].length;
            }
        }
        if (lnGain) lnGain[i] = lg;
        if (endPoint)
            for (int d = 0; d < 3; ++d) endPoint[3 * size_t(i) + d] = x[d];
        status[i] = fail < 0 ? 0 : 1;
    }
    return 0;
}

}  // extern "C"
