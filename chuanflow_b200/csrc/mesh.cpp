// Host mesh: block generation, addressing checks and geometry.
//
// The geometry must be bit-identical to the reference's polyMesh, so every
// quantity below is evaluated with the same IEEE operations in the same order
// as src/3d/src/mesh/polyMesh.cpp:83-288 (this file is compiled with
// -ffp-contract=off so no multiply-add is fused).  The block generator emits
// the face order that BlockMesh::create's first-registration deduplication
// produces (src/3d/src/mesh/blockMesh.cpp:76-185), derived in closed form
// instead of through a face map.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <unordered_map>

#include "cfg_internal.h"

namespace cfg
{
namespace
{

inline double dot(const Vec& a, const Vec& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Vec cross(const Vec& a, const Vec& b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double mag(const Vec& a) { return std::sqrt(dot(a, a)); }

}  // namespace

Mesh blockMesh(const Vec& mn, const Vec& mx, int64_t nx, int64_t ny, int64_t nz,
               const std::vector<std::string>& names, const std::vector<std::string>& types)
{
    if (nx <= 0 || ny <= 0 || nz <= 0) fail(CFG_EMESH, "blockMesh: cell counts must be positive");
    Mesh m;
    m.bnx = nx;
    m.bny = ny;
    m.bnz = nz;
    m.bmin = mn;
    m.bmax = mx;
    auto pid = [&](int64_t i, int64_t j, int64_t k) { return i + (nx + 1) * (j + (ny + 1) * k); };
    m.points.resize(static_cast<size_t>((nx + 1) * (ny + 1) * (nz + 1)));
    for (int64_t k = 0; k <= nz; ++k)
        for (int64_t j = 0; j <= ny; ++j)
            for (int64_t i = 0; i <= nx; ++i)
                m.points[static_cast<size_t>(pid(i, j, k))] = {
                    mn.x + (mx.x - mn.x) * static_cast<double>(i) / static_cast<double>(nx),
                    mn.y + (mx.y - mn.y) * static_cast<double>(j) / static_cast<double>(ny),
                    mn.z + (mx.z - mn.z) * static_cast<double>(k) / static_cast<double>(nz)};

    // A hex face is registered first by the lower-numbered of its two cells,
    // and cells are visited in id order with faces zlo zhi ylo yhi xlo xhi.
    // So at cell (i,j,k) the new faces are: zlo iff k==0, zhi always, ylo iff
    // j==0, yhi always, xlo iff i==0, xhi always; a new face is internal iff
    // the cell across it exists.  Boundary faces then go to their side's list.
    const int64_t nInt = (nx - 1) * ny * nz + nx * (ny - 1) * nz + nx * ny * (nz - 1);
    const int64_t nBnd = 2 * (ny * nz + nx * nz + nx * ny);
    std::vector<int64_t> intVerts;
    intVerts.reserve(static_cast<size_t>(4 * nInt));
    m.owner.reserve(static_cast<size_t>(nInt + nBnd));
    m.neighbour.reserve(static_cast<size_t>(nInt));
    std::vector<int64_t> sideVerts[6], sideOwner[6];
    for (int64_t k = 0; k < nz; ++k)
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i)
            {
                const int64_t c = i + nx * (j + ny * k);
                const int64_t v0 = pid(i, j, k), v1 = pid(i + 1, j, k), v2 = pid(i + 1, j + 1, k),
                              v3 = pid(i, j + 1, k), v4 = pid(i, j, k + 1), v5 = pid(i + 1, j, k + 1),
                              v6 = pid(i + 1, j + 1, k + 1), v7 = pid(i, j + 1, k + 1);
                struct Kind
                {
                    int64_t v[4];
                    bool isNew;
                    int64_t other;  // -1: boundary
                    int side;
                };
                const Kind kinds[6] = {
                    {{v0, v1, v2, v3}, k == 0, -1, 4},
                    {{v4, v5, v6, v7}, true, k + 1 < nz ? c + nx * ny : -1, 5},
                    {{v0, v1, v5, v4}, j == 0, -1, 2},
                    {{v2, v3, v7, v6}, true, j + 1 < ny ? c + nx : -1, 3},
                    {{v0, v3, v7, v4}, i == 0, -1, 0},
                    {{v1, v2, v6, v5}, true, i + 1 < nx ? c + 1 : -1, 1}};
                for (const Kind& kd : kinds)
                {
                    if (!kd.isNew) continue;
                    if (kd.other >= 0)
                    {
                        intVerts.insert(intVerts.end(), kd.v, kd.v + 4);
                        m.owner.push_back(c);
                        m.neighbour.push_back(kd.other);
                    }
                    else
                    {
                        sideVerts[kd.side].insert(sideVerts[kd.side].end(), kd.v, kd.v + 4);
                        sideOwner[kd.side].push_back(c);
                    }
                }
            }
    m.faceVerts = std::move(intVerts);
    for (int s = 0; s < 6; ++s)
    {
        if (sideOwner[s].empty()) continue;
        Mesh::Patch p;
        p.name = names[static_cast<size_t>(s)];
        p.type = types[static_cast<size_t>(s)];
        p.start = static_cast<int64_t>(m.owner.size());
        p.size = static_cast<int64_t>(sideOwner[s].size());
        m.faceVerts.insert(m.faceVerts.end(), sideVerts[s].begin(), sideVerts[s].end());
        m.owner.insert(m.owner.end(), sideOwner[s].begin(), sideOwner[s].end());
        m.patches.push_back(std::move(p));
    }
    m.faceOffsets.resize(m.owner.size() + 1);
    for (size_t f = 0; f <= m.owner.size(); ++f) m.faceOffsets[f] = static_cast<int64_t>(4 * f);
    m.finish();
    return m;
}

namespace
{
/// faces (or cells) per thread chunk in the geometry loops
constexpr int64_t kFaceChunk = 1 << 15;
}  // namespace

void Mesh::finish()
{
    const int64_t nF = nFaces(), nI = nInternal();
    if (static_cast<int64_t>(faceOffsets.size()) != nF + 1) fail(CFG_EMESH, "polyMesh: face offsets size");
    // polyMesh.cpp:23 counts cells from the owners alone; a cell that owns
    // no face (every face shared with lower-numbered cells, possible in
    // element meshes) would then index past the cell arrays there, so the
    // neighbours are counted too (identical whenever the reference is defined)
    nCells = 0;
    for (int64_t o : owner) nCells = std::max(nCells, o + 1);
    for (int64_t nb : neighbour) nCells = std::max(nCells, nb + 1);
    parallelChunks(nF, kFaceChunk, [&](int64_t fb, int64_t fe) {
        for (int64_t f = fb; f < fe; ++f)
        {
            if (faceOffsets[f + 1] - faceOffsets[f] < 3) fail(CFG_EMESH, "polyMesh: face with fewer than 3 vertices");
            if (owner[f] < 0) fail(CFG_EMESH, "polyMesh: negative owner");
            for (int64_t q = faceOffsets[f]; q < faceOffsets[f + 1]; ++q)
                if (faceVerts[q] < 0 || faceVerts[q] >= static_cast<int64_t>(points.size()))
                    fail(CFG_EMESH, "polyMesh: face vertex out of range");
            if (f < nI && (neighbour[f] < 0 || neighbour[f] >= nCells))
                fail(CFG_EMESH, "polyMesh: neighbour out of range at face " + std::to_string(f));
        }
    });
    // face -> patch, patches must cover every boundary face exactly once
    // (polyMesh.cpp:35-61)
    facePatch.assign(static_cast<size_t>(nF), -1);
    for (size_t i = 0; i < patches.size(); ++i)
    {
        const Patch& p = patches[i];
        for (int64_t f = p.start; f < p.start + p.size; ++f)
        {
            if (f < nI) fail(CFG_EMESH, "polyMesh: patch '" + p.name + "' covers internal face " + std::to_string(f));
            if (f >= nF) fail(CFG_EMESH, "polyMesh: patch '" + p.name + "' beyond the last face");
            if (facePatch[static_cast<size_t>(f)] >= 0)
                fail(CFG_EMESH, "polyMesh: boundary face " + std::to_string(f) + " in two patches");
            facePatch[static_cast<size_t>(f)] = static_cast<int64_t>(i);
        }
    }
    for (int64_t f = nI; f < nF; ++f)
        if (facePatch[static_cast<size_t>(f)] < 0)
            fail(CFG_EMESH, "polyMesh: boundary face " + std::to_string(f) + " is not in any patch");
    calcGeometry();
}

void Mesh::calcGeometry()
{
    const int64_t nF = nFaces(), nI = nInternal();
    Cf.assign(static_cast<size_t>(nF), Vec{});
    Sf.assign(static_cast<size_t>(nF), Vec{});
    auto P = [&](int64_t v) -> const Vec& { return points[static_cast<size_t>(v)]; };

    // Per-face and per-cell steps run on the host's threads; the sums over
    // a cell's faces stay serial, in face order, so every value is the one
    // the serial loops give.
    // fan-triangle area vectors and face centroids
    parallelChunks(nF, kFaceChunk, [&](int64_t fb, int64_t fe) {
    for (int64_t f = fb; f < fe; ++f)
    {
        const int64_t* vs = faceVerts.data() + faceOffsets[f];
        const int64_t nv = faceOffsets[f + 1] - faceOffsets[f];
        const Vec v0 = P(vs[0]);
        Vec n{};
        for (int64_t i = 1; i + 1 < nv; ++i) n = n + cross(P(vs[i]) - v0, P(vs[i + 1]) - v0);
        Sf[static_cast<size_t>(f)] = n * 0.5;
        bool exactMean = nv == 3;
        if (nv == 4)
        {
            const Vec a = P(vs[0]) + P(vs[2]), b = P(vs[1]) + P(vs[3]);
            exactMean = a.x == b.x && a.y == b.y && a.z == b.z;
        }
        Vec c{};
        const double wSum = exactMean ? 0.0 : dot(n, n);
        if (!exactMean && wSum > 0)
        {
            for (int64_t i = 1; i + 1 < nv; ++i)
            {
                const Vec vi = P(vs[i]), vj = P(vs[i + 1]);
                const double w = dot(cross(vi - v0, vj - v0), n);
                c = c + (v0 + vi + vj) * w;
            }
            Cf[static_cast<size_t>(f)] = c / (3.0 * wSum);
        }
        else
        {
            for (int64_t i = 0; i < nv; ++i) c = c + P(vs[i]);
            Cf[static_cast<size_t>(f)] = c / static_cast<double>(nv);
        }
    }
    });

    // provisional cell centres (mean of face centres), used only to orient
    std::vector<Vec> est(static_cast<size_t>(nCells));
    std::vector<int64_t> cnt(static_cast<size_t>(nCells), 0);
    for (int64_t f = 0; f < nF; ++f)
    {
        const size_t o = static_cast<size_t>(owner[f]);
        est[o] = est[o] + Cf[static_cast<size_t>(f)];
        ++cnt[o];
        if (f < nI)
        {
            const size_t nb = static_cast<size_t>(neighbour[f]);
            est[nb] = est[nb] + Cf[static_cast<size_t>(f)];
            ++cnt[nb];
        }
    }
    for (size_t c = 0; c < est.size(); ++c)
        if (cnt[c] > 0) est[c] = est[c] / static_cast<double>(cnt[c]);
    magSf.resize(static_cast<size_t>(nF));
    parallelChunks(nF, kFaceChunk, [&](int64_t fb, int64_t fe) {
        for (int64_t f = fb; f < fe; ++f)
        {
            const size_t o = static_cast<size_t>(owner[f]);
            const Vec dd = f < nI ? est[static_cast<size_t>(neighbour[f])] - est[o] : Cf[static_cast<size_t>(f)] - est[o];
            Vec& sf = Sf[static_cast<size_t>(f)];
            const double side = dot(sf, dd);
            const double tol = 1e-12 * mag(sf) * mag(dd);
            if (side < -tol) sf = Vec{-sf.x, -sf.y, -sf.z};
            magSf[static_cast<size_t>(f)] = mag(sf);
        }
    });

    // volumes and centroids through the divergence theorem over fan tets
    V.assign(static_cast<size_t>(nCells), 0.0);
    C.assign(static_cast<size_t>(nCells), Vec{});
    std::vector<Vec> moment(static_cast<size_t>(nCells));
    std::vector<double> faceV(static_cast<size_t>(nF));
    std::vector<Vec> faceM(static_cast<size_t>(nF));
    parallelChunks(nF, kFaceChunk, [&](int64_t fb, int64_t fe) {
    for (int64_t f = fb; f < fe; ++f)
    {
        const int64_t* vs = faceVerts.data() + faceOffsets[f];
        const int64_t nv = faceOffsets[f + 1] - faceOffsets[f];
        const Vec v0 = P(vs[0]);
        double fv = 0;
        Vec fm{}, raw{};
        for (int64_t i = 1; i + 1 < nv; ++i)
        {
            const Vec a = P(vs[i]) - v0, b = P(vs[i + 1]) - v0;
            const double tV = dot(v0, cross(a, b)) / 6.0;
            fv += tV;
            fm = fm + ((v0 + P(vs[i]) + P(vs[i + 1])) / 4.0) * tV;
        }
        for (int64_t i = 1; i + 1 < nv; ++i) raw = raw + cross(P(vs[i]) - v0, P(vs[i + 1]) - v0);
        const double s = dot(raw, Sf[static_cast<size_t>(f)]) >= 0 ? 1.0 : -1.0;
        faceV[static_cast<size_t>(f)] = s * fv;
        faceM[static_cast<size_t>(f)] = fm * s;
    }
    });
    for (int64_t f = 0; f < nF; ++f)
    {
        const size_t o = static_cast<size_t>(owner[f]);
        V[o] += faceV[static_cast<size_t>(f)];
        moment[o] = moment[o] + faceM[static_cast<size_t>(f)];
        if (f < nI)
        {
            const size_t nb = static_cast<size_t>(neighbour[f]);
            V[nb] -= faceV[static_cast<size_t>(f)];
            moment[nb] = moment[nb] - faceM[static_cast<size_t>(f)];
        }
    }
    parallelChunks(nCells, kFaceChunk, [&](int64_t cb, int64_t ce) {
        for (int64_t c = cb; c < ce; ++c)
        {
            C[c] = moment[c] / V[c];
            V[c] = std::abs(V[c]);
            if (!(V[c] > 0)) fail(CFG_EMESH, "polyMesh: degenerate cell volume for cell " + std::to_string(c));
        }
    });
    d.resize(static_cast<size_t>(nF));
    invDist.resize(static_cast<size_t>(nF));
    parallelChunks(nF, kFaceChunk, [&](int64_t fb, int64_t fe) {
        for (int64_t f = fb; f < fe; ++f)
        {
            const size_t o = static_cast<size_t>(owner[f]);
            d[static_cast<size_t>(f)] = f < nI ? C[static_cast<size_t>(neighbour[f])] - C[o] : Cf[static_cast<size_t>(f)] - C[o];
            const double dm = mag(d[static_cast<size_t>(f)]);
            if (!(dm > 0)) fail(CFG_EMESH, "polyMesh: zero owner-neighbour distance at face " + std::to_string(f));
            invDist[static_cast<size_t>(f)] = 1.0 / dm;
        }
    });
}

std::vector<double> Mesh::ownerWeights() const
{
    // makeInternalOwnerWeights (interpolate.cpp:15-35): 1 - clamp(t, 0, 1),
    // t the owner-to-face-centre projection on d over |d|^2
    const int64_t nI = nInternal();
    std::vector<double> w(static_cast<size_t>(std::max<int64_t>(1, nI)), 0.5);
    for (int64_t f = 0; f < nI; ++f)
    {
        const Vec& dd = d[static_cast<size_t>(f)];
        const double t = dot(Cf[static_cast<size_t>(f)] - C[static_cast<size_t>(owner[f])], dd) / dot(dd, dd);
        const double tc = t < 0.0 ? 0.0 : (1.0 < t ? 1.0 : t);
        w[static_cast<size_t>(f)] = 1.0 - tc;
    }
    return w;
}

std::vector<Vec> Mesh::skewVectors(const std::vector<double>& ow) const
{
    // makeFaceSkewVectors (interpolate.cpp:37-48)
    std::vector<Vec> s(static_cast<size_t>(nFaces()));
    for (int64_t f = 0; f < nInternal(); ++f)
    {
        const Vec& co = C[static_cast<size_t>(owner[f])];
        const Vec& cn = C[static_cast<size_t>(neighbour[f])];
        s[static_cast<size_t>(f)] = Cf[static_cast<size_t>(f)] - (co + (cn - co) * (1.0 - ow[static_cast<size_t>(f)]));
    }
    return s;
}

}  // namespace cfg

namespace cfg
{
namespace
{

/// Local face rings of the gmsh volume elements (tet 4, hex 5, prism 6),
/// in the order src/3d/src/mesh/gmshMesh.cpp:52-68 registers them.
const std::vector<std::vector<int>>& faceRings(int type)
{
    static const std::vector<std::vector<int>> tet = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    static const std::vector<std::vector<int>> hex = {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 1, 5, 4},
                                                      {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}};
    static const std::vector<std::vector<int>> prism = {{0, 1, 2}, {3, 4, 5}, {0, 1, 4, 3}, {1, 2, 5, 4}, {2, 0, 3, 5}};
    static const std::vector<std::vector<int>> none;
    switch (type)
    {
    case 4: return tet;
    case 5: return hex;
    case 6: return prism;
    default: return none;
    }
}

}  // namespace

Mesh meshFromCells(const std::vector<Vec>& points, const std::vector<int32_t>& types,
                   const std::vector<int64_t>& cellOffsets, const std::vector<int64_t>& cellVerts)
{
    return meshFromCells(points, types, cellOffsets, cellVerts, {}, {});
}

Mesh meshFromCells(const std::vector<Vec>& points, const std::vector<int32_t>& types,
                   const std::vector<int64_t>& cellOffsets, const std::vector<int64_t>& cellVerts,
                   const SurfaceNames& surfaceNames, const std::map<std::string, std::string>& patchTypes)
{
    // faces registered cell by cell in each element's ring order and
    // deduplicated by their sorted vertices; the first registration keeps
    // its vertex ring (gmshMesh.cpp:578-607)
    struct Ref
    {
        int64_t v0, nv, cell0, cell1;
    };
    const int64_t nCells = static_cast<int64_t>(types.size());
    const int64_t nPoints = static_cast<int64_t>(points.size());
    std::vector<int64_t> ringVerts;
    std::vector<Ref> refs;
    // every registration (cell c, ring k) is filed under its smallest
    // vertex.  Threads own ranges of vertices: each walks all registrations
    // in order, files those of its own vertices and finds for each the
    // first registration with the same key in that vertex's short bucket.
    // A serial walk then numbers the faces in order of first registration.
    std::vector<int64_t> regStart(static_cast<size_t>(nCells) + 1, 0);
    for (int64_t c = 0; c < nCells; ++c)
    {
        const auto& rings = faceRings(types[static_cast<size_t>(c)]);
        if (rings.empty()) fail(CFG_EMESH, "mesh: cell type " + std::to_string(types[c]) + " is not tet (4), hex (5) or prism (6)");
        const int64_t need = types[c] == 4 ? 4 : (types[c] == 5 ? 8 : 6);
        if (cellOffsets[c + 1] - cellOffsets[c] != need) fail(CFG_EMESH, "mesh: cell vertex count does not fit its type");
        const int64_t* cv = cellVerts.data() + cellOffsets[c];
        for (int64_t k = 0; k < need; ++k)
            if (cv[k] < 0 || cv[k] >= nPoints) fail(CFG_EMESH, "mesh: cell vertex out of range");
        regStart[c + 1] = regStart[c] + static_cast<int64_t>(rings.size());
    }
    const int64_t nReg = regStart[nCells];
    // first[r]: the earliest registration with r's key (r itself if none)
    std::vector<int64_t> first(static_cast<size_t>(nReg));
    {
        std::vector<int64_t> bucket(static_cast<size_t>(nPoints) + 1, 0);
        const int64_t hw = std::max<int64_t>(1, std::thread::hardware_concurrency());
        const int64_t parts = std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(hw, 32), nReg / (1 << 16)));
        auto forOwn = [&](int64_t part, auto&& fn) {
            const int64_t vlo = nPoints * part / parts, vhi = nPoints * (part + 1) / parts;
            for (int64_t c = 0; c < nCells; ++c)
            {
                const int64_t* cv = cellVerts.data() + cellOffsets[c];
                int64_t r = regStart[c];
                for (const auto& ring : faceRings(types[static_cast<size_t>(c)]))
                {
                    int64_t lo = cv[ring[0]];
                    for (size_t k = 1; k < ring.size(); ++k) lo = std::min(lo, cv[ring[k]]);
                    if (lo >= vlo && lo < vhi) fn(r, cv, ring, lo);
                    ++r;
                }
            }
        };
        parallelChunks(parts, 1, [&](int64_t pb, int64_t pe) {
            for (int64_t part = pb; part < pe; ++part)
                forOwn(part, [&](int64_t, const int64_t*, const std::vector<int>&, int64_t lo) { ++bucket[static_cast<size_t>(lo) + 1]; });
        });
        for (int64_t v = 0; v < nPoints; ++v) bucket[v + 1] += bucket[v];
        struct Slot
        {
            int64_t k1, k2, k3, reg;  // the sorted key after its smallest vertex (-1 padded)
        };
        std::vector<Slot> slots(static_cast<size_t>(bucket[nPoints]));
        std::vector<int64_t> fill(bucket.begin(), bucket.end() - 1);
        parallelChunks(parts, 1, [&](int64_t pb, int64_t pe) {
            for (int64_t part = pb; part < pe; ++part)
                forOwn(part, [&](int64_t r, const int64_t* cv, const std::vector<int>& ring, int64_t lo) {
                    std::array<int64_t, 4> key{-1, -1, -1, -1};
                    for (size_t k = 0; k < ring.size(); ++k) key[k] = cv[ring[k]];
                    std::sort(key.begin(), key.begin() + static_cast<long>(ring.size()));
                    const size_t b = static_cast<size_t>(lo);
                    for (int64_t q = bucket[b]; q < fill[b]; ++q)
                    {
                        const Slot& sl = slots[static_cast<size_t>(q)];
                        if (sl.k1 == key[1] && sl.k2 == key[2] && sl.k3 == key[3])
                        {
                            first[static_cast<size_t>(r)] = sl.reg;
                            return;
                        }
                    }
                    slots[static_cast<size_t>(fill[b]++)] = {key[1], key[2], key[3], r};
                    first[static_cast<size_t>(r)] = r;
                });
        });
    }
    ringVerts.reserve(static_cast<size_t>(4 * 4 * nCells));
    refs.reserve(static_cast<size_t>(4 * nCells));
    for (int64_t c = 0; c < nCells; ++c)
    {
        const int64_t* cv = cellVerts.data() + cellOffsets[c];
        int64_t r = regStart[c];
        for (const auto& ring : faceRings(types[static_cast<size_t>(c)]))
        {
            const int64_t f0 = first[static_cast<size_t>(r)];
            if (f0 == r)
            {
                first[static_cast<size_t>(r)] = ~static_cast<int64_t>(refs.size());  // now the face index
                refs.push_back({static_cast<int64_t>(ringVerts.size()), static_cast<int64_t>(ring.size()), c, -1});
                for (int k : ring) ringVerts.push_back(cv[k]);
            }
            else
            {
                Ref& fr = refs[static_cast<size_t>(~first[static_cast<size_t>(f0)])];
                if (fr.cell1 != -1) fail(CFG_EMESH, "mesh: a face belongs to three cells: the mesh is not manifold");
                fr.cell1 = c;
            }
            ++r;
        }
    }
    std::vector<int64_t>().swap(first);
    // ---- boundary faces to patches ----
    // A boundary face takes the physical-group name of a surface element on
    // it, else the name of the bounding-box plane it lies in: within 1e-9 of
    // the box's largest extent of that plane.  Every point is on one side of
    // a box plane, so the face vertex farthest from it decides, and each
    // face's per-axis coordinate range is enough: fmax - lo <= eps puts it
    // in a low plane, hi - fmin <= eps in a high one.  Planes are tried in
    // the order low x, high x, low y, high y, low z, high z.
    double lo[3] = {points[0].x, points[0].y, points[0].z};
    double hi[3] = {lo[0], lo[1], lo[2]};
    {
        const int64_t parts = std::max<int64_t>(1, std::min<int64_t>(32, nPoints / (1 << 16)));
        std::vector<std::array<double, 6>> part(static_cast<size_t>(parts));
        parallelChunks(parts, 1, [&](int64_t pb, int64_t pe) {
            for (int64_t q = pb; q < pe; ++q)
            {
                auto& box = part[static_cast<size_t>(q)];
                box = {lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]};
                for (int64_t i = nPoints * q / parts; i < nPoints * (q + 1) / parts; ++i)
                {
                    const double x[3] = {points[i].x, points[i].y, points[i].z};
                    for (int d = 0; d < 3; ++d)
                    {
                        box[d] = std::min(box[d], x[d]);
                        box[3 + d] = std::max(box[3 + d], x[d]);
                    }
                }
            }
        });
        for (const auto& box : part)
            for (int d = 0; d < 3; ++d)
            {
                lo[d] = std::min(lo[d], box[d]);
                hi[d] = std::max(hi[d], box[3 + d]);
            }
    }
    const double eps = 1e-9 * std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1e-300});
    static const char* const kPlane[6] = {"xmin", "xmax", "ymin", "ymax", "zmin", "zmax"};
    auto boxPlane = [&](const Ref& r) -> int {
        double fmin[3], fmax[3];
        for (int64_t k = 0; k < r.nv; ++k)
        {
            const Vec& v = points[static_cast<size_t>(ringVerts[r.v0 + k])];
            const double x[3] = {v.x, v.y, v.z};
            for (int d = 0; d < 3; ++d)
            {
                fmin[d] = k ? std::min(fmin[d], x[d]) : x[d];
                fmax[d] = k ? std::max(fmax[d], x[d]) : x[d];
            }
        }
        for (int d = 0; d < 3; ++d)
        {
            if (fmax[d] - lo[d] <= eps) return 2 * d;
            if (hi[d] - fmin[d] <= eps) return 2 * d + 1;
        }
        return -1;
    };
    // the group of a face: a surface element with the face's vertex set, or
    // for a quad one with the vertex set left when one ring vertex (0, then
    // 1, 2, 3) is dropped -- a triangulated surface splits quads in two
    auto surfaceGroup = [&](const Ref& r) -> const std::string* {
        std::array<int64_t, 5> key;
        key.fill(-1);
        std::copy(ringVerts.begin() + r.v0, ringVerts.begin() + r.v0 + r.nv, key.begin());
        std::sort(key.begin(), key.begin() + r.nv);
        if (const auto it = surfaceNames.find(key); it != surfaceNames.end()) return &it->second;
        if (r.nv != 4) return nullptr;
        for (int drop = 0; drop < 4; ++drop)
        {
            const int64_t gone = ringVerts[r.v0 + drop];
            std::array<int64_t, 5> tri;
            tri.fill(-1);
            bool dropped = false;
            for (int k = 0, t = 0; k < 4; ++k)
            {
                if (!dropped && key[k] == gone)
                {
                    dropped = true;
                    continue;
                }
                tri[t++] = key[k];
            }
            if (const auto it = surfaceNames.find(tri); it != surfaceNames.end()) return &it->second;
        }
        return nullptr;
    };
    Mesh m;
    m.points = points;
    // patches in order of their first face
    std::vector<std::vector<size_t>> patchFaces;
    std::unordered_map<std::string, size_t> patchOf;
    std::vector<size_t> internal;
    for (size_t i = 0; i < refs.size(); ++i)
    {
        Ref& r = refs[i];
        if (r.cell1 != -1)
        {
            if (r.cell0 > r.cell1) std::swap(r.cell0, r.cell1);
            internal.push_back(i);
            continue;
        }
        const std::string* group = surfaceNames.empty() ? nullptr : surfaceGroup(r);
        std::string name;
        if (group) name = *group;
        else
        {
            const int plane = boxPlane(r);
            if (plane < 0)
            {
                std::string list;
                for (int64_t k = 0; k < r.nv; ++k) list += " " + std::to_string(ringVerts[r.v0 + k]);
                fail(CFG_EMESH, "gmsh: boundary face with nodes" + list +
                                    " belongs to no physical group and lies on no bounding-box plane; give every "
                                    "boundary surface a physical group in Gmsh");
            }
            name = kPlane[plane];
        }
        auto [it, added] = patchOf.emplace(name, m.patches.size());
        if (added)
        {
            Mesh::Patch p;
            p.name = name;
            const auto t = patchTypes.find(name);
            p.type = t != patchTypes.end() ? t->second : "wall";
            m.patches.push_back(p);
            patchFaces.emplace_back();
        }
        patchFaces[it->second].push_back(i);
    }
    m.faceOffsets.reserve(refs.size() + 1);
    m.faceVerts.reserve(ringVerts.size());
    m.owner.reserve(refs.size());
    m.neighbour.reserve(internal.size());
    m.faceOffsets.push_back(0);
    auto addFace = [&](const Ref& r) {
        for (int64_t k = 0; k < r.nv; ++k) m.faceVerts.push_back(ringVerts[r.v0 + k]);
        m.faceOffsets.push_back(static_cast<int64_t>(m.faceVerts.size()));
        m.owner.push_back(r.cell0);
    };
    for (size_t i : internal)
    {
        addFace(refs[i]);
        m.neighbour.push_back(refs[i].cell1);
    }
    for (size_t pi = 0; pi < patchFaces.size(); ++pi)
    {
        m.patches[pi].start = static_cast<int64_t>(m.owner.size());  // in order of first appearance
        m.patches[pi].size = static_cast<int64_t>(patchFaces[pi].size());
        for (size_t i : patchFaces[pi]) addFace(refs[i]);
    }
    m.finish();
    return m;
}

}  // namespace cfg

// ---------------------------------------------------------------------------
// Device cell numbering (no reference counterpart: the reference keeps the
// mesh's own order, and its only reordering is the domain decomposition's
// coordinate median split, domainDecomposition.cpp:27-77).  Renumbering
// changes where each cell's values sit in device memory, never the order of
// any sum: per-cell face lists and matrix rows keep the original face and
// column order, so results are bit-identical in every numbering.
// ---------------------------------------------------------------------------
namespace cfg
{

CellGraph cellGraph(const Mesh& M)
{
    const int64_t nC = M.nCells, nI = M.nInternal();
    CellGraph g;
    g.start.assign(static_cast<size_t>(nC) + 1, 0);
    for (int64_t f = 0; f < nI; ++f)
    {
        ++g.start[M.owner[f] + 1];
        ++g.start[M.neighbour[f] + 1];
    }
    for (int64_t c = 0; c < nC; ++c) g.start[c + 1] += g.start[c];
    std::vector<int64_t> fill(g.start.begin(), g.start.end() - 1);
    g.adj.resize(static_cast<size_t>(g.start[nC]));
    for (int64_t f = 0; f < nI; ++f)
    {
        const int64_t o = M.owner[f], n = M.neighbour[f];
        g.adj[fill[o]++] = n;
        g.adj[fill[n]++] = o;
    }
    // distinct neighbours in ascending order (two faces may join one pair)
    std::vector<int64_t> s2(static_cast<size_t>(nC) + 1, 0);
    size_t w = 0;
    for (int64_t c = 0; c < nC; ++c)
    {
        auto b = g.adj.begin() + g.start[c], e = g.adj.begin() + g.start[c + 1];
        std::sort(b, e);
        const auto u = std::unique(b, e);
        for (auto it = b; it != u; ++it) g.adj[w++] = *it;
        s2[c + 1] = static_cast<int64_t>(w);
    }
    g.adj.resize(w);
    g.start.swap(s2);
    return g;
}

std::vector<int> greedyColours(const CellGraph& g, int* nColours)
{
    const int64_t nC = static_cast<int64_t>(g.start.size()) - 1;
    std::vector<int> colour(static_cast<size_t>(nC), -1), mark(static_cast<size_t>(nC) + 2, -1);
    int nCol = 0;
    for (int64_t c = 0; c < nC; ++c)
    {
        for (int64_t k = g.start[c]; k < g.start[c + 1]; ++k)
        {
            const int cj = colour[g.adj[k]];
            if (cj >= 0) mark[cj] = static_cast<int>(c);
        }
        int col = 0;
        while (mark[col] == c) ++col;
        colour[c] = col;
        nCol = std::max(nCol, col + 1);
    }
    if (nColours) *nColours = nCol;
    return colour;
}

namespace
{

/// Breadth-first levels from `root` over cells not yet numbered; returns the
/// eccentricity and leaves the last level in `last`.
int bfsLevels(const CellGraph& g, int64_t root, const std::vector<char>& numbered, std::vector<int64_t>& stamp,
              int64_t tag, std::vector<int64_t>& last)
{
    std::vector<int64_t> cur{root}, next;
    stamp[root] = tag;
    int ecc = 0;
    for (;;)
    {
        next.clear();
        for (int64_t u : cur)
            for (int64_t k = g.start[u]; k < g.start[u + 1]; ++k)
            {
                const int64_t v = g.adj[k];
                if (numbered[v] || stamp[v] == tag) continue;
                stamp[v] = tag;
                next.push_back(v);
            }
        if (next.empty()) break;
        cur.swap(next);
        ++ecc;
    }
    last = cur;
    return ecc;
}

}  // namespace

/// Reverse Cuthill-McKee (Cuthill & McKee 1969; reversed, George 1971).
/// Each connected component starts from a pseudo-peripheral cell (George &
/// Liu 1979, at most 8 rounds): the unnumbered cell of least (degree, index),
/// moved to the least-(degree, index) cell of its farthest level while that
/// increases the eccentricity.  Cells are numbered breadth-first, each
/// cell's unnumbered neighbours by increasing (degree, index); the whole
/// sequence is then reversed.  Returns new -> old.
std::vector<int64_t> rcmOrder(const CellGraph& g)
{
    const int64_t nC = static_cast<int64_t>(g.start.size()) - 1;
    auto deg = [&](int64_t c) { return g.start[c + 1] - g.start[c]; };
    auto less = [&](int64_t a, int64_t b) { return deg(a) != deg(b) ? deg(a) < deg(b) : a < b; };
    std::vector<int64_t> byDeg(static_cast<size_t>(nC));
    for (int64_t c = 0; c < nC; ++c) byDeg[c] = c;
    std::stable_sort(byDeg.begin(), byDeg.end(), less);
    std::vector<char> numbered(static_cast<size_t>(nC), 0);
    std::vector<int64_t> stamp(static_cast<size_t>(nC), -1), order, last, last2, nb;
    order.reserve(static_cast<size_t>(nC));
    int64_t tag = 0;
    size_t scan = 0;
    while (static_cast<int64_t>(order.size()) < nC)
    {
        while (numbered[byDeg[scan]]) ++scan;
        int64_t root = byDeg[scan];
        int ecc = bfsLevels(g, root, numbered, stamp, tag++, last);
        for (int round = 0; round < 8; ++round)
        {
            int64_t cand = last[0];
            for (int64_t v : last)
                if (less(v, cand)) cand = v;
            const int ecc2 = bfsLevels(g, cand, numbered, stamp, tag++, last2);
            if (ecc2 <= ecc) break;
            root = cand;
            ecc = ecc2;
            last.swap(last2);
        }
        size_t head = order.size();
        order.push_back(root);
        numbered[root] = 1;
        while (head < order.size())
        {
            const int64_t u = order[head++];
            nb.clear();
            for (int64_t k = g.start[u]; k < g.start[u + 1]; ++k)
                if (!numbered[g.adj[k]]) nb.push_back(g.adj[k]);
            std::sort(nb.begin(), nb.end(), less);
            for (int64_t v : nb)
            {
                numbered[v] = 1;
                order.push_back(v);
            }
        }
    }
    std::reverse(order.begin(), order.end());
    return order;
}

int defaultCellOrder()
{
    if (const char* e = std::getenv("CHUANFLOW_CELL_ORDER"))
    {
        const std::string s(e);
        if (s == "identity") return CFG_ORDER_IDENTITY;
        if (s == "colour") return CFG_ORDER_COLOUR;
        if (s == "rcm") return CFG_ORDER_RCM;
        if (s == "rcm-colour") return CFG_ORDER_RCM_COLOUR;
    }
    return CFG_ORDER_IDENTITY;
}

std::vector<int64_t> cellOrder(const Mesh& M, int mode)
{
    if (mode == CFG_ORDER_DEFAULT) mode = defaultCellOrder();
    const int64_t nC = M.nCells;
    std::vector<int64_t> order(static_cast<size_t>(nC));
    for (int64_t c = 0; c < nC; ++c) order[c] = c;
    if (mode == CFG_ORDER_IDENTITY) return order;
    if (mode != CFG_ORDER_COLOUR && mode != CFG_ORDER_RCM && mode != CFG_ORDER_RCM_COLOUR)
        fail(CFG_EINVAL, "unknown cell order " + std::to_string(mode));
    const CellGraph g = cellGraph(M);
    if (mode == CFG_ORDER_RCM || mode == CFG_ORDER_RCM_COLOUR) order = rcmOrder(g);
    if (mode == CFG_ORDER_COLOUR || mode == CFG_ORDER_RCM_COLOUR)
    {
        // colour blocks, each in the base order: the colour of a cell is its
        // greedy colour in the original numbering
        const std::vector<int> colour = greedyColours(g, nullptr);
        std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return colour[a] < colour[b]; });
    }
    return order;
}

}  // namespace cfg
