// Internal declarations shared by the host C++ and the CUDA sources of
// libchuanflow_b200.so.
#pragma once

#include <algorithm>
#include <cstdint>
#include <exception>
#include <stdexcept>
#include <array>
#include <thread>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

#include "chuanflow_b200.h"

namespace cfg
{

/// Error carried to the C boundary as a status code + message.
struct Error : std::runtime_error
{
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void fail(int code, const std::string& msg) { throw Error(code, msg); }

/// Sets the calling thread's message for cfg_last_error (api.cpp).
void setLastError(const std::string& msg);

/// Runs fn(begin, end) over [0, n) in contiguous chunks of at least
/// `minChunk` items on the host's threads.  Chunks must be independent;
/// if any throw, the exception of the lowest such chunk is rethrown, which
/// is the one a serial loop would have met first.
template <class F>
void parallelChunks(int64_t n, int64_t minChunk, F&& fn)
{
    const int64_t hw = std::max<int64_t>(1, std::thread::hardware_concurrency());
    const int64_t t = std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(hw, 32), n / std::max<int64_t>(1, minChunk)));
    if (t == 1)
    {
        if (n > 0) fn(int64_t(0), n);
        return;
    }
    std::vector<std::exception_ptr> err(static_cast<size_t>(t));
    std::vector<std::thread> th;
    th.reserve(static_cast<size_t>(t));
    for (int64_t k = 0; k < t; ++k)
        th.emplace_back([&, k] {
            try
            {
                fn(n * k / t, n * (k + 1) / t);
            }
            catch (...)
            {
                err[static_cast<size_t>(k)] = std::current_exception();
            }
        });
    for (auto& x : th) x.join();
    for (const auto& e : err)
        if (e) std::rethrow_exception(e);
}

struct Vec
{
    double x = 0, y = 0, z = 0;
};

inline Vec operator+(const Vec& a, const Vec& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec operator-(const Vec& a, const Vec& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec operator*(const Vec& a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline Vec operator/(const Vec& a, double s) { return {a.x / s, a.y / s, a.z / s}; }

/// Host mesh: the reference polyMesh's addressing plus its geometry,
/// computed in the reference's operation order (polyMesh.cpp:83-288).
struct Mesh
{
    std::vector<Vec> points;
    std::vector<int64_t> faceOffsets, faceVerts, owner, neighbour;
    struct Patch
    {
        std::string name, type;
        int64_t start = 0, size = 0;
    };
    std::vector<Patch> patches;
    int64_t nCells = 0;

    // block-structured origin (for the interior jitter helper); nx < 0 if none
    int64_t bnx = -1, bny = -1, bnz = -1;
    Vec bmin, bmax;

    // geometry
    std::vector<double> V;
    std::vector<Vec> C, Cf, Sf, d;
    std::vector<double> magSf, invDist;
    std::vector<int64_t> facePatch;

    int64_t nFaces() const { return static_cast<int64_t>(owner.size()); }
    int64_t nInternal() const { return static_cast<int64_t>(neighbour.size()); }
    int64_t nBoundary() const { return nFaces() - nInternal(); }

    void finish();       // addressing checks + geometry
    void calcGeometry();
    std::vector<double> ownerWeights() const;  // size max(1, nInt)
    std::vector<Vec> skewVectors(const std::vector<double>& ow) const;
};

/// polyMesh from volume cells as the reference's gmsh reader builds it
/// (types: 4 tet, 5 hex, 6 prism; boundary patches named after the
/// bounding-box planes).
Mesh meshFromCells(const std::vector<Vec>& points, const std::vector<int32_t>& types,
                   const std::vector<int64_t>& cellOffsets, const std::vector<int64_t>& cellVerts);

/// sorted vertex key of a face (unused slots -1) -> physical-group name
struct FaceKeyHash
{
    size_t operator()(const std::array<int64_t, 5>& k) const
    {
        uint64_t h = 1469598103934665603ULL;
        for (int64_t v : k)
        {
            h ^= static_cast<uint64_t>(v) + 0x9E3779B97F4A7C15ULL;
            h *= 1099511628211ULL;
            h ^= h >> 31;
        }
        return static_cast<size_t>(h);
    }
};
using SurfaceNames = std::unordered_map<std::array<int64_t, 5>, std::string, FaceKeyHash>;
/// the same with boundary faces named by their surface element's physical
/// group when there is one, and patch types from `patchTypes` (else "wall")
Mesh meshFromCells(const std::vector<Vec>& points, const std::vector<int32_t>& types,
                   const std::vector<int64_t>& cellOffsets, const std::vector<int64_t>& cellVerts,
                   const SurfaceNames& surfaceNames, const std::map<std::string, std::string>& patchTypes);

/// a cell field for writeVtu: nComp 1 or 3, cell-major, original order
struct VtuField
{
    std::string name;
    int nComp;
    std::vector<double> data;
};
/// VtkWriter::write (vtkWrite.cpp:33-131): scalars then vectors, each in the
/// order given; binary = raw appended arrays instead of ASCII
void writeVtu(const Mesh& M, const std::string& path, const std::vector<VtuField>& fields, bool binary);
/// writeFieldsHdf5's file (hdf5Write.cpp:38-95): /points, /owner,
/// /neighbour and /fields/<name> (one f64 per cell), by this library's own
/// HDF5 encoder (hdf5.cpp)
void writeHdf5(const Mesh& M, const std::string& path, const std::vector<std::pair<std::string, const double*>>& fields);

/// GmshMesh::fromFile (gmshMesh.cpp:534-776): ASCII .msh 2.2 or 4.x
Mesh readGmsh(const std::string& path, const std::map<std::string, std::string>& patchTypes);

Mesh blockMesh(const Vec& mn, const Vec& mx, int64_t nx, int64_t ny, int64_t nz,
               const std::vector<std::string>& names, const std::vector<std::string>& types);

/// Distinct cell neighbours across internal faces, ascending, as a CSR.
struct CellGraph
{
    std::vector<int64_t> start, adj;
};
CellGraph cellGraph(const Mesh& M);
/// First-fit colours in ascending cell order (no two neighbours alike).
std::vector<int> greedyColours(const CellGraph& g, int* nColours);
/// Reverse Cuthill-McKee order, new -> old.
std::vector<int64_t> rcmOrder(const CellGraph& g);
/// The device numbering of a cfg_cell_order mode, new -> old.
std::vector<int64_t> cellOrder(const Mesh& M, int mode);

}  // namespace cfg

struct cfg_mesh
{
    cfg::Mesh m;
};
