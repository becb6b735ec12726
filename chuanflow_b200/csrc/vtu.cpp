// VTK XML unstructured-grid output of a mesh and its cell fields, as the
// reference's VtkWriter writes it (src/3d/src/io/vtkWrite.cpp:33-131): every
// cell a polyhedron (type 42) whose connectivity is its vertices in the
// order its faces (ascending face index, polyMesh::cells) first visit them,
// plus the VTK face stream.  ASCII output is byte-identical to the
// reference's (12 significant digits); the binary form writes the same
// arrays raw in an appended block (UInt64 headers, little endian), with the
// face offsets VTK readers need for polyhedra, at memory speed.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "cfg_internal.h"

namespace cfg
{
namespace
{

struct Topo
{
    std::vector<int64_t> conn, offsets, faces, faceOffsets;
};

Topo topology(const Mesh& M)
{
    const int64_t nC = M.nCells, nF = M.nFaces(), nI = M.nInternal();
    // each cell's faces in ascending face order (polyMesh::cells)
    std::vector<int64_t> cStart(static_cast<size_t>(nC) + 1, 0), cFaces;
    for (int64_t f = 0; f < nF; ++f)
    {
        ++cStart[static_cast<size_t>(M.owner[f]) + 1];
        if (f < nI) ++cStart[static_cast<size_t>(M.neighbour[f]) + 1];
    }
    for (int64_t c = 0; c < nC; ++c) cStart[c + 1] += cStart[c];
    cFaces.resize(static_cast<size_t>(cStart[nC]));
    {
        std::vector<int64_t> fill(cStart.begin(), cStart.end() - 1);
        for (int64_t f = 0; f < nF; ++f)
        {
            cFaces[static_cast<size_t>(fill[static_cast<size_t>(M.owner[f])]++)] = f;
            if (f < nI) cFaces[static_cast<size_t>(fill[static_cast<size_t>(M.neighbour[f])]++)] = f;
        }
    }
    // a cell's vertices in the order its faces first visit them; cells are
    // independent, so two parallel passes: sizes, then the arrays at their
    // prefix offsets
    auto cellVerts = [&](int64_t c, std::vector<int64_t>& verts) {
        verts.clear();
        for (int64_t q = cStart[c]; q < cStart[c + 1]; ++q)
        {
            const int64_t f = cFaces[static_cast<size_t>(q)];
            for (int64_t k = M.faceOffsets[f]; k < M.faceOffsets[f + 1]; ++k)
            {
                const int64_t v = M.faceVerts[k];
                bool seen = false;
                for (int64_t w : verts) seen = seen || w == v;
                if (!seen) verts.push_back(v);
            }
        }
    };
    constexpr int64_t kChunk = 1 << 14;
    std::vector<int64_t> nConn(static_cast<size_t>(nC) + 1, 0), nFaceStream(static_cast<size_t>(nC) + 1, 0);
    parallelChunks(nC, kChunk, [&](int64_t cb, int64_t ce) {
        std::vector<int64_t> verts;
        for (int64_t c = cb; c < ce; ++c)
        {
            cellVerts(c, verts);
            nConn[c + 1] = static_cast<int64_t>(verts.size());
            int64_t len = 1;
            for (int64_t q = cStart[c]; q < cStart[c + 1]; ++q)
            {
                const int64_t f = cFaces[static_cast<size_t>(q)];
                len += 1 + M.faceOffsets[f + 1] - M.faceOffsets[f];
            }
            nFaceStream[c + 1] = len;
        }
    });
    for (int64_t c = 0; c < nC; ++c)
    {
        nConn[c + 1] += nConn[c];
        nFaceStream[c + 1] += nFaceStream[c];
    }
    Topo t;
    t.conn.resize(static_cast<size_t>(nConn[nC]));
    t.faces.resize(static_cast<size_t>(nFaceStream[nC]));
    t.offsets.assign(nConn.begin() + 1, nConn.end());
    t.faceOffsets.assign(nFaceStream.begin() + 1, nFaceStream.end());
    parallelChunks(nC, kChunk, [&](int64_t cb, int64_t ce) {
        std::vector<int64_t> verts;
        for (int64_t c = cb; c < ce; ++c)
        {
            cellVerts(c, verts);
            std::copy(verts.begin(), verts.end(), t.conn.begin() + nConn[c]);
            int64_t w = nFaceStream[c];
            t.faces[static_cast<size_t>(w++)] = cStart[c + 1] - cStart[c];
            for (int64_t q = cStart[c]; q < cStart[c + 1]; ++q)
            {
                const int64_t f = cFaces[static_cast<size_t>(q)];
                t.faces[static_cast<size_t>(w++)] = M.faceOffsets[f + 1] - M.faceOffsets[f];
                for (int64_t k = M.faceOffsets[f]; k < M.faceOffsets[f + 1]; ++k) t.faces[static_cast<size_t>(w++)] = M.faceVerts[k];
            }
        }
    });
    return t;
}

std::string g12(double v)
{
    char b[40];
    std::snprintf(b, sizeof b, "%.12g", v);
    return b;
}

}  // namespace

void writeVtu(const Mesh& M, const std::string& path, const std::vector<VtuField>& fields, bool binary)
{
    std::FILE* fp = std::fopen(path.c_str(), "wb");
    if (!fp) fail(CFG_EINVAL, "vtk: cannot open '" + path + "' for writing");
    const Topo t = topology(M);
    const int64_t nP = static_cast<int64_t>(M.points.size()), nC = M.nCells;
    std::string h = "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\"";
    if (binary) h += " header_type=\"UInt64\"";
    h += ">\n<UnstructuredGrid>\n<Piece NumberOfPoints=\"" + std::to_string(nP) + "\" NumberOfCells=\"" +
         std::to_string(nC) + "\">\n";
    if (!binary)
    {
        std::string s = h;
        s.reserve(static_cast<size_t>(nP) * 60 + t.conn.size() * 8 + t.faces.size() * 8);
        s += "<Points>\n<DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n";
        for (const Vec& p : M.points) s += g12(p.x) + ' ' + g12(p.y) + ' ' + g12(p.z) + '\n';
        s += "</DataArray>\n</Points>\n<Cells>\n<DataArray type=\"Int64\" Name=\"connectivity\" format=\"ascii\">\n";
        int64_t prev = 0;
        for (int64_t c = 0; c < nC; ++c)
        {
            for (int64_t k = prev; k < t.offsets[c]; ++k) s += std::to_string(t.conn[k]) + ' ';
            s += '\n';
            prev = t.offsets[c];
        }
        s += "</DataArray>\n<DataArray type=\"Int64\" Name=\"offsets\" format=\"ascii\">\n";
        for (int64_t o : t.offsets) s += std::to_string(o) + ' ';
        s += "</DataArray>\n<DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n";
        for (int64_t c = 0; c < nC; ++c) s += "42 ";
        s += "</DataArray>\n<DataArray type=\"Int64\" Name=\"faces\" format=\"ascii\">\n";
        prev = 0;
        for (int64_t c = 0; c < nC; ++c)
        {
            for (int64_t k = prev; k < t.faceOffsets[c]; ++k) s += std::to_string(t.faces[k]) + ' ';
            s += '\n';
            prev = t.faceOffsets[c];
        }
        s += "</DataArray>\n</Cells>\n";
        if (!fields.empty())
        {
            s += "<CellData>\n";
            for (int pass = 0; pass < 2; ++pass)  // the scalars, then the vectors
                for (const VtuField& f : fields)
                {
                    if ((f.nComp == 3) != (pass == 1)) continue;
                    s += "<DataArray type=\"Float64\" Name=\"" + f.name + "\"" +
                         (f.nComp == 3 ? std::string(" NumberOfComponents=\"3\"") : std::string()) +
                         " format=\"ascii\">\n";
                    for (int64_t c = 0; c < nC; ++c)
                    {
                        for (int q = 0; q < f.nComp; ++q)
                        {
                            if (q) s += ' ';
                            s += g12(f.data[static_cast<size_t>(c * f.nComp + q)]);
                        }
                        s += '\n';
                    }
                    s += "</DataArray>\n";
                }
            s += "</CellData>\n";
        }
        s += "</Piece>\n</UnstructuredGrid>\n</VTKFile>\n";
        const size_t w = std::fwrite(s.data(), 1, s.size(), fp);
        std::fclose(fp);
        if (w != s.size()) fail(CFG_EINVAL, "vtk: short write to '" + path + "'");
        return;
    }
    // binary: every array raw in one appended block
    struct Block
    {
        const void* p;
        uint64_t bytes;
    };
    std::vector<Block> blocks;
    std::vector<double> pts(3 * static_cast<size_t>(nP));
    for (int64_t i = 0; i < nP; ++i)
    {
        pts[3 * i] = M.points[i].x;
        pts[3 * i + 1] = M.points[i].y;
        pts[3 * i + 2] = M.points[i].z;
    }
    std::vector<uint8_t> types(static_cast<size_t>(nC), 42);
    uint64_t off = 0;
    std::string s = h;
    auto arr = [&](const char* type, const std::string& name, int nComp, const void* p, uint64_t bytes) {
        s += std::string("<DataArray type=\"") + type + "\"" + (name.empty() ? "" : " Name=\"" + name + "\"") +
             (nComp > 1 ? " NumberOfComponents=\"" + std::to_string(nComp) + "\"" : std::string()) +
             " format=\"appended\" offset=\"" + std::to_string(off) + "\"/>\n";
        blocks.push_back({p, bytes});
        off += 8 + bytes;
    };
    s += "<Points>\n";
    arr("Float64", "", 3, pts.data(), pts.size() * 8);
    s += "</Points>\n<Cells>\n";
    arr("Int64", "connectivity", 1, t.conn.data(), t.conn.size() * 8);
    arr("Int64", "offsets", 1, t.offsets.data(), t.offsets.size() * 8);
    arr("UInt8", "types", 1, types.data(), types.size());
    arr("Int64", "faces", 1, t.faces.data(), t.faces.size() * 8);
    arr("Int64", "faceoffsets", 1, t.faceOffsets.data(), t.faceOffsets.size() * 8);
    s += "</Cells>\n";
    if (!fields.empty())
    {
        s += "<CellData>\n";
        for (int pass = 0; pass < 2; ++pass)
            for (const VtuField& f : fields)
                if ((f.nComp == 3) == (pass == 1)) arr("Float64", f.name, f.nComp, f.data.data(), f.data.size() * 8);
        s += "</CellData>\n";
    }
    s += "</Piece>\n</UnstructuredGrid>\n<AppendedData encoding=\"raw\">\n_";
    bool ok = std::fwrite(s.data(), 1, s.size(), fp) == s.size();
    for (const Block& b : blocks)
    {
        ok = ok && std::fwrite(&b.bytes, 8, 1, fp) == 1;
        ok = ok && (b.bytes == 0 || std::fwrite(b.p, 1, b.bytes, fp) == b.bytes);
    }
    const char* tail = "\n</AppendedData>\n</VTKFile>\n";
    ok = ok && std::fwrite(tail, 1, std::strlen(tail), fp) == std::strlen(tail);
    std::fclose(fp);
    if (!ok) fail(CFG_EINVAL, "vtk: short write to '" + path + "'");
}

}  // namespace cfg
