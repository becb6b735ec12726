// HDF5 output of a mesh and its cell fields with the layout of the
// reference's writeFieldsHdf5 (src/3d/src/io/hdf5Write.cpp:38-95):
// /points (nPoints x 3 f64), /owner and /neighbour (int64, one per face) and
// a group /fields of one 1-D f64 dataset per cell field.  The reference
// needs the HDF5 C library (and refuses to write without it); this encoder
// writes the file format itself, in its oldest and most widely read form:
// superblock version 0, symbol-table groups (version-1 B-tree of group
// nodes, local heap of link names, symbol-table nodes), version-1 object
// headers and contiguous little-endian datasets.  Link names in a group are
// kept in strcmp order, as the format's group B-tree requires.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "cfg_internal.h"

namespace cfg
{
namespace
{

constexpr uint64_t kUndef = ~uint64_t(0);   // the format's undefined address
constexpr uint64_t kHeapFreeNone = 1;       // local heap: no free block
constexpr int kLeafK = 4;                   // symbol-table node holds up to 2K entries
constexpr int kInternalK = 16;              // group B-tree node holds up to 2K children
constexpr uint64_t kSuperblock = 96;
constexpr uint64_t kEntry = 40;             // symbol-table entry, 8-byte offsets
constexpr uint64_t kSnod = 8 + 2 * kLeafK * kEntry;
constexpr uint64_t kTree = 24 + (2 * kInternalK + 1) * 8 + 2 * kInternalK * 8;
constexpr uint64_t kGroupHeader = 16 + 8 + 16;  // prefix + symbol-table message

uint64_t pad8(uint64_t n) { return (n + 7) & ~uint64_t(7); }

/// little-endian byte sink with absolute-position checks
struct Sink
{
    explicit Sink(std::FILE* f) : fp(f) {}
    std::FILE* fp;
    uint64_t pos = 0;
    std::vector<unsigned char> buf;

    void u8(unsigned v) { buf.push_back(static_cast<unsigned char>(v)); }
    void le(uint64_t v, int n)
    {
        for (int i = 0; i < n; ++i) buf.push_back(static_cast<unsigned char>(v >> (8 * i)));
    }
    void zeros(uint64_t n) { buf.insert(buf.end(), static_cast<size_t>(n), 0); }
    void text(const std::string& s) { buf.insert(buf.end(), s.begin(), s.end()); }
    void flush(const std::string& path)
    {
        if (!buf.empty() && std::fwrite(buf.data(), 1, buf.size(), fp) != buf.size())
            fail(CFG_EINVAL, "hdf5: cannot write '" + path + "'");
        pos += buf.size();
        buf.clear();
    }
    /// the next byte written lands at `at`
    void expect(uint64_t at) const
    {
        if (pos + buf.size() != at) fail(CFG_EINVAL, "hdf5: internal layout error");
    }
    void raw(const void* p, uint64_t n, const std::string& path)
    {
        flush(path);
        if (n > 0 && std::fwrite(p, 1, static_cast<size_t>(n), fp) != n)
            fail(CFG_EINVAL, "hdf5: cannot write '" + path + "'");
        pos += n;
    }
};

struct Dataset
{
    std::string name;
    int rank;
    uint64_t dims[2];
    bool real;  // f64, else int64
    const void* data;
    uint64_t header = 0, addr = 0;

    uint64_t bytes() const { return 8 * dims[0] * (rank == 2 ? dims[1] : 1); }
    uint64_t headerSize() const
    {
        return 16 + (8 + 8 + 8 * static_cast<uint64_t>(rank)) + (8 + (real ? 24 : 16)) + (8 + 8) + (8 + 24);
    }
};

/// one symbol-table group: its links (datasets or one subgroup) by name
struct Group
{
    struct Link
    {
        std::string name;
        uint64_t header;
        bool group;
        uint64_t tree, heap;  // a subgroup's cached addresses
    };
    std::vector<Link> links;
    uint64_t header = 0, heap = 0, heapData = 0, tree = 0, snods = 0;
    std::vector<uint64_t> nameOffset;
    uint64_t heapSize = 0;

    size_t nSnods() const { return (links.size() + 2 * kLeafK - 1) / (2 * kLeafK); }
    uint64_t size() const { return kGroupHeader + 32 + heapSize + kTree + nSnods() * kSnod; }
    void layoutNames()
    {
        std::sort(links.begin(), links.end(), [](const Link& a, const Link& b) {
            return std::strcmp(a.name.c_str(), b.name.c_str()) < 0;
        });
        nameOffset.clear();
        uint64_t off = 8;  // offset 0 holds the empty name
        for (const Link& l : links)
        {
            nameOffset.push_back(off);
            off += pad8(l.name.size() + 1);
        }
        heapSize = off;
    }
    void place(uint64_t at)
    {
        header = at;
        heap = header + kGroupHeader;
        heapData = heap + 32;
        tree = heapData + heapSize;
        snods = tree + kTree;
    }
};

void objectHeaderPrefix(Sink& s, int nMessages, uint64_t messageBytes)
{
    s.u8(1);  // version
    s.u8(0);
    s.le(static_cast<uint64_t>(nMessages), 2);
    s.le(1, 4);  // reference count
    s.le(messageBytes, 4);
    s.zeros(4);  // alignment of the first message
}

void message(Sink& s, unsigned type, uint64_t size, unsigned flags)
{
    s.le(type, 2);
    s.le(size, 2);
    s.u8(flags);
    s.zeros(3);
}

void writeGroup(Sink& s, const Group& g)
{
    s.expect(g.header);
    objectHeaderPrefix(s, 1, 8 + 16);
    message(s, 0x0011, 16, 0);  // symbol table: B-tree, local heap
    s.le(g.tree, 8);
    s.le(g.heap, 8);

    s.expect(g.heap);
    s.text("HEAP");
    s.u8(0);
    s.zeros(3);
    s.le(g.heapSize, 8);
    s.le(kHeapFreeNone, 8);
    s.le(g.heapData, 8);
    s.zeros(8);
    for (size_t i = 0; i < g.links.size(); ++i)
    {
        s.text(g.links[i].name);
        s.zeros(pad8(g.links[i].name.size() + 1) - g.links[i].name.size());
    }

    s.expect(g.tree);
    const size_t nS = g.nSnods();
    s.text("TREE");
    s.u8(0);  // group node
    s.u8(0);  // leaf level
    s.le(nS, 2);
    s.le(kUndef, 8);
    s.le(kUndef, 8);
    s.le(0, 8);  // key 0: the empty name
    for (size_t k = 0; k < nS; ++k)
    {
        const size_t last = std::min(g.links.size(), (k + 1) * 2 * kLeafK) - 1;
        s.le(g.snods + k * kSnod, 8);
        s.le(g.nameOffset[last], 8);  // the largest name in child k
    }
    s.zeros(kTree - (24 + 8 + 16 * nS));

    for (size_t k = 0; k < nS; ++k)
    {
        s.expect(g.snods + k * kSnod);
        const size_t b = k * 2 * kLeafK, e = std::min(g.links.size(), b + 2 * kLeafK);
        s.text("SNOD");
        s.u8(1);
        s.u8(0);
        s.le(e - b, 2);
        for (size_t i = b; i < e; ++i)
        {
            const Group::Link& l = g.links[i];
            s.le(g.nameOffset[i], 8);
            s.le(l.header, 8);
            s.le(l.group ? 1 : 0, 4);  // cache type: a group caches its B-tree and heap
            s.zeros(4);
            if (l.group)
            {
                s.le(l.tree, 8);
                s.le(l.heap, 8);
            }
            else
            {
                s.zeros(16);
            }
        }
        s.zeros(kSnod - 8 - (e - b) * kEntry);
    }
}

void writeDataset(Sink& s, const Dataset& d, const std::string& path)
{
    s.expect(d.header);
    objectHeaderPrefix(s, 4, d.headerSize() - 16);
    // dataspace, version 1
    message(s, 0x0001, 8 + 8 * static_cast<uint64_t>(d.rank), 0);
    s.u8(1);
    s.u8(static_cast<unsigned>(d.rank));
    s.u8(0);  // no maximum dimensions
    s.zeros(5);
    for (int r = 0; r < d.rank; ++r) s.le(d.dims[r], 8);
    // datatype, version 1: IEEE f64 or signed int64, little endian
    if (d.real)
    {
        message(s, 0x0003, 24, 1);
        s.u8(0x11);  // class 1 (floating point), version 1
        s.u8(0x20);  // implied mantissa msb, little endian, zero padding
        s.u8(63);    // sign bit
        s.u8(0);
        s.le(8, 4);
        s.le(0, 2);   // bit offset
        s.le(64, 2);  // precision
        s.u8(52);     // exponent location
        s.u8(11);     // exponent size
        s.u8(0);      // mantissa location
        s.u8(52);     // mantissa size
        s.le(1023, 4);
        s.zeros(4);
    }
    else
    {
        message(s, 0x0003, 16, 1);
        s.u8(0x10);  // class 0 (fixed point), version 1
        s.u8(0x08);  // signed, little endian
        s.u8(0);
        s.u8(0);
        s.le(8, 4);
        s.le(0, 2);
        s.le(64, 2);
        s.zeros(4);
    }
    // fill value, version 2: allocated late, written if set, none defined
    message(s, 0x0005, 8, 1);
    s.u8(2);
    s.u8(2);
    s.u8(2);
    s.u8(0);
    s.zeros(4);
    // layout, version 3: contiguous
    message(s, 0x0008, 24, 0);
    s.u8(3);
    s.u8(1);
    s.le(d.bytes() > 0 ? d.addr : kUndef, 8);
    s.le(d.bytes(), 8);
    s.zeros(6);
    s.expect(d.header + d.headerSize());
    s.raw(d.data, d.bytes(), path);
}

}  // namespace

void writeHdf5(const Mesh& M, const std::string& path, const std::vector<std::pair<std::string, const double*>>& fields)
{
    for (const auto& f : fields)
    {
        const std::string& n = f.first;
        if (n.empty() || n == "." || n.find('/') != std::string::npos)
            fail(CFG_EINVAL, "hdf5: cannot create dataset '" + n + "'");
    }
    for (size_t i = 0; i < fields.size(); ++i)
        for (size_t j = i + 1; j < fields.size(); ++j)
            if (fields[i].first == fields[j].first) fail(CFG_EINVAL, "hdf5: field '" + fields[i].first + "' given twice");
    if (fields.size() > static_cast<size_t>(2 * kLeafK * 2 * kInternalK))
        fail(CFG_EINVAL, "hdf5: at most " + std::to_string(2 * kLeafK * 2 * kInternalK) + " fields per file");

    const uint64_t nP = M.points.size(), nF = static_cast<uint64_t>(M.nFaces()), nI = static_cast<uint64_t>(M.nInternal());
    std::vector<Dataset> top = {{"points", 2, {nP, 3}, true, M.points.data()},
                                {"owner", 1, {nF, 0}, false, M.owner.data()},
                                {"neighbour", 1, {nI, 0}, false, M.neighbour.data()}};
    std::vector<Dataset> cells;
    for (const auto& f : fields) cells.push_back({f.first, 1, {static_cast<uint64_t>(M.nCells), 0}, true, f.second});

    // addresses: superblock, root group, its datasets, /fields, its datasets
    Group root, sub;
    root.links = {{"points", 0, false, 0, 0}, {"owner", 0, false, 0, 0}, {"neighbour", 0, false, 0, 0},
                  {"fields", 0, true, 0, 0}};
    for (const auto& d : cells) sub.links.push_back({d.name, 0, false, 0, 0});
    root.layoutNames();
    sub.layoutNames();
    uint64_t at = kSuperblock;
    root.place(at);
    at += root.size();
    for (Dataset& d : top)
    {
        d.header = at;
        d.addr = at + d.headerSize();
        at = d.addr + d.bytes();
    }
    sub.place(at);
    at += sub.size();
    for (Dataset& d : cells)
    {
        d.header = at;
        d.addr = at + d.headerSize();
        at = d.addr + d.bytes();
    }
    const uint64_t eof = at;
    auto headerOf = [](const std::vector<Dataset>& ds, const std::string& n) {
        for (const Dataset& d : ds)
            if (d.name == n) return d.header;
        return kUndef;
    };
    for (Group::Link& l : root.links)
    {
        if (l.group)
        {
            l.header = sub.header;
            l.tree = sub.tree;
            l.heap = sub.heap;
        }
        else
        {
            l.header = headerOf(top, l.name);
        }
    }
    for (Group::Link& l : sub.links) l.header = headerOf(cells, l.name);

    std::FILE* fp = std::fopen(path.c_str(), "wb");
    if (!fp) fail(CFG_EINVAL, "hdf5: cannot open '" + path + "' for writing");
    Sink s(fp);
    try
    {
        // superblock, version 0
        const unsigned char sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
        for (unsigned char c : sig) s.u8(c);
        s.u8(0);  // superblock
        s.u8(0);  // free-space storage
        s.u8(0);  // root group symbol table entry
        s.u8(0);
        s.u8(0);  // shared header messages
        s.u8(8);  // size of offsets
        s.u8(8);  // size of lengths
        s.u8(0);
        s.le(kLeafK, 2);
        s.le(kInternalK, 2);
        s.le(0, 4);  // consistency flags
        s.le(0, 8);  // base address
        s.le(kUndef, 8);
        s.le(eof, 8);
        s.le(kUndef, 8);
        // root group symbol table entry, caching its B-tree and heap
        s.le(0, 8);
        s.le(root.header, 8);
        s.le(1, 4);
        s.zeros(4);
        s.le(root.tree, 8);
        s.le(root.heap, 8);
        writeGroup(s, root);
        for (const Dataset& d : top) writeDataset(s, d, path);
        writeGroup(s, sub);
        for (const Dataset& d : cells) writeDataset(s, d, path);
        s.flush(path);
        if (s.pos != eof) fail(CFG_EINVAL, "hdf5: internal layout error");
    }
    catch (...)
    {
        std::fclose(fp);
        throw;
    }
    if (std::fclose(fp) != 0) fail(CFG_EINVAL, "hdf5: cannot write '" + path + "'");
}

}  // namespace cfg
