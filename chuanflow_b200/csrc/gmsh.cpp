// GmshMesh::fromFile (src/3d/src/mesh/gmshMesh.cpp:534-776): ASCII .msh 2.2
// and 4.x with first-order tetrahedra, hexahedra and prisms; boundary faces
// named by the physical groups of the surface elements (a quad face also by
// one of its triangles), else by the bounding-box plane they lie on.
//
// The file is read into memory once and tokenised row by row in place
// (string views, strtol/strtod), so a multi-million-element file parses at
// memory speed instead of through one std::string per token.  The reading
// rules follow the reference: the section layout and header checks, the
// 4.x node blocks with or without tag lists, per-block element tags, node
// tags renumbered densely in ascending order, and its error messages.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <string_view>
#include <charconv>
#include <unordered_map>
#include <vector>

#include "cfg_internal.h"

namespace cfg
{
namespace
{

/// the tokens of one row: a view into its section's flat token array
class Row
{
public:
    Row() = default;
    Row(const std::string_view* b, size_t n) : b_(b), n_(n) {}
    size_t size() const { return n_; }
    bool empty() const { return n_ == 0; }
    const std::string_view& operator[](size_t i) const { return b_[i]; }

private:
    const std::string_view* b_ = nullptr;
    size_t n_ = 0;
};

int nodesPerElement(int type)
{
    switch (type)
    {
    case 1: return 2;
    case 2: return 3;
    case 3: return 4;
    case 4: return 4;
    case 5: return 8;
    case 6: return 6;
    case 7: return 5;
    default: return 0;
    }
}

long toInt(std::string_view t, const char* where)
{
    {
        // the common case without a copy: the whole token is the number
        long v = 0;
        const char* b = t.data();
        const char* e = b + t.size();
        if (b < e && *b == '+') ++b;
        const auto r = std::from_chars(b, e, v);
        if (r.ec == std::errc() && r.ptr == e) return v;
    }
    std::string s(t);
    char* end = nullptr;
    errno = 0;
    const long v = std::strtol(s.c_str(), &end, 10);
    if (end == s.c_str() || errno) fail(CFG_EMESH, "gmsh: expected an integer but found '" + s + "' in " + where);
    return v;
}

double toDouble(std::string_view t, const char* where)
{
    {
        // from_chars rounds correctly, as strtod does
        double v = 0;
        const char* b = t.data();
        const char* e = b + t.size();
        if (b < e && *b == '+') ++b;
        const auto r = std::from_chars(b, e, v);
        if (r.ec == std::errc() && r.ptr == e) return v;
    }
    std::string s(t);
    char* end = nullptr;
    const double v = std::strtod(s.c_str(), &end);
    if (end == s.c_str()) fail(CFG_EMESH, "gmsh: expected a number but found '" + s + "' in " + where);
    return v;
}

bool isIntegerToken(std::string_view t) { return t.find_first_of(".eE") == std::string_view::npos; }

/// the non-empty rows of one $Name ... $EndName section
class Section
{
public:
    Section() = default;
    /// rows over `tokens` (kept here, so the rows' views stay valid)
    Section(std::vector<std::string_view> tokens, const std::vector<size_t>& start, std::string where)
        : tok_(std::move(tokens)), where_(std::move(where))
    {
        rows_.reserve(start.empty() ? 0 : start.size() - 1);
        for (size_t k = 0; k + 1 < start.size(); ++k) rows_.emplace_back(tok_.data() + start[k], start[k + 1] - start[k]);
    }
    Section(Section&&) = default;
    Section& operator=(Section&&) = default;
    Section(const Section&) = delete;
    Section& operator=(const Section&) = delete;
    bool found() const { return !rows_.empty(); }
    bool atEnd() const { return pos_ >= rows_.size(); }
    const Row& take()
    {
        if (atEnd())
            fail(CFG_EMESH, "gmsh: truncated file: " + where_ + " ends after " + std::to_string(rows_.size()) + " rows");
        return rows_[pos_++];
    }
    size_t remaining() const { return rows_.size() - pos_; }
    /// row k after the current one, not consumed (k < remaining())
    const Row& peek(size_t k) const { return rows_[pos_ + k]; }
    void skip(size_t n) { pos_ += n; }
    bool takeSingleInt(long& v)
    {
        if (atEnd() || rows_[pos_].size() != 1 || !isIntegerToken(rows_[pos_][0])) return false;
        v = toInt(rows_[pos_][0], where_.c_str());
        ++pos_;
        return true;
    }

private:
    std::vector<std::string_view> tok_;
    std::vector<Row> rows_;
    size_t pos_ = 0;
    std::string where_;
};

struct File
{
    std::string text;
    std::vector<std::pair<size_t, size_t>> lines;  // [begin, end) of every line
    std::vector<size_t> marks;                     // the lines whose first token starts with '$'

    /// appends the tokens of line li; returns how many
    size_t tokens(size_t li, std::vector<std::string_view>& out) const
    {
        const size_t before = out.size();
        const char* s = text.data() + lines[li].first;
        const char* e = text.data() + lines[li].second;
        while (s < e)
        {
            while (s < e && (*s == ' ' || *s == '\t' || *s == '\r' || *s == '\v' || *s == '\f')) ++s;
            const char* b = s;
            while (s < e && !(*s == ' ' || *s == '\t' || *s == '\r' || *s == '\v' || *s == '\f')) ++s;
            if (s > b) out.emplace_back(b, static_cast<size_t>(s - b));
        }
        return out.size() - before;
    }

    std::string_view first(size_t li) const
    {
        const char* s = text.data() + lines[li].first;
        const char* e = text.data() + lines[li].second;
        while (s < e && std::isspace(static_cast<unsigned char>(*s))) ++s;
        const char* b = s;
        while (s < e && !std::isspace(static_cast<unsigned char>(*s))) ++s;
        return std::string_view(b, static_cast<size_t>(s - b));
    }

    Section section(const std::string& name, const std::string& path, bool required) const
    {
        // only the '$' lines can open or close a section
        const std::string begin = "$" + name, end = "$End" + name;
        for (size_t mi = 0; mi < marks.size(); ++mi)
        {
            const size_t i = marks[mi];
            if (first(i) != begin) continue;
            for (size_t mj = mi + 1; mj < marks.size(); ++mj)
            {
                const size_t j = marks[mj];
                if (first(j) != end) continue;
                // lines tokenized in parallel chunks, then joined in order
                const int64_t nl = static_cast<int64_t>(j - i - 1);
                const int64_t parts = std::max<int64_t>(1, std::min<int64_t>(64, nl / 8192));
                std::vector<std::vector<std::string_view>> ptok(static_cast<size_t>(parts));
                std::vector<std::vector<size_t>> pend(static_cast<size_t>(parts));
                parallelChunks(parts, 1, [&](int64_t pb, int64_t pe) {
                    for (int64_t q = pb; q < pe; ++q)
                    {
                        auto& tq = ptok[static_cast<size_t>(q)];
                        auto& eq = pend[static_cast<size_t>(q)];
                        const size_t lb = i + 1 + static_cast<size_t>(nl * q / parts);
                        const size_t le = i + 1 + static_cast<size_t>(nl * (q + 1) / parts);
                        eq.reserve(le - lb);
                        for (size_t k = lb; k < le; ++k)
                            if (tokens(k, tq) > 0) eq.push_back(tq.size());  // empty lines make no row
                    }
                });
                std::vector<size_t> tokBase(static_cast<size_t>(parts) + 1, 0), rowBase(static_cast<size_t>(parts) + 1, 0);
                for (size_t q = 0; q < static_cast<size_t>(parts); ++q)
                {
                    tokBase[q + 1] = tokBase[q] + ptok[q].size();
                    rowBase[q + 1] = rowBase[q] + pend[q].size();
                }
                std::vector<std::string_view> tok(tokBase.back());
                std::vector<size_t> start(rowBase.back() + 1, 0);
                parallelChunks(parts, 1, [&](int64_t pb, int64_t pe) {
                    for (int64_t q = pb; q < pe; ++q)
                    {
                        const size_t u = static_cast<size_t>(q);
                        std::copy(ptok[u].begin(), ptok[u].end(), tok.begin() + static_cast<long>(tokBase[u]));
                        for (size_t r = 0; r < pend[u].size(); ++r) start[rowBase[u] + r + 1] = tokBase[u] + pend[u][r];
                        std::vector<std::string_view>().swap(ptok[u]);
                    }
                });
                return Section(std::move(tok), start, begin + " in " + path);
            }
            fail(CFG_EMESH, "gmsh: section " + begin + " in " + path + " is not terminated");
        }
        if (required) fail(CFG_EMESH, "gmsh: " + path + " has no " + begin + " section");
        return Section();
    }
};

struct Element
{
    int type;
    long physical;
    std::vector<int64_t> nodes;
};

}  // namespace

Mesh readGmsh(const std::string& path, const std::map<std::string, std::string>& patchTypes)
{
    File f;
    {
        std::FILE* fp = std::fopen(path.c_str(), "rb");
        if (!fp) fail(CFG_EMESH, "gmsh: cannot open " + path);
        std::fseek(fp, 0, SEEK_END);
        const long size = std::ftell(fp);
        std::fseek(fp, 0, SEEK_SET);
        f.text.resize(static_cast<size_t>(std::max(size, 0L)));
        const size_t got = size > 0 ? std::fread(&f.text[0], 1, static_cast<size_t>(size), fp) : 0;
        std::fclose(fp);
        if (got != f.text.size()) fail(CFG_EMESH, "gmsh: cannot read " + path);
        size_t b = 0;
        const char* t = f.text.data();
        const size_t n = f.text.size();
        while (b <= n)
        {
            const void* nl = b < n ? std::memchr(t + b, '\n', n - b) : nullptr;
            const size_t i = nl ? static_cast<size_t>(static_cast<const char*>(nl) - t) : n;
            if (i < n || i > b)
            {
                size_t k = b;
                while (k < i && std::isspace(static_cast<unsigned char>(t[k]))) ++k;
                if (k < i && t[k] == '$') f.marks.push_back(f.lines.size());
                f.lines.push_back({b, i});
            }
            b = i + 1;
        }
    }

    Section fmt = f.section("MeshFormat", path, true);
    const Row& fv = fmt.take();
    if (fv.size() < 2) fail(CFG_EMESH, "gmsh: malformed $MeshFormat in " + path);
    const double version = toDouble(fv[0], "$MeshFormat");
    if (toInt(fv[1], "$MeshFormat") != 0)
        fail(CFG_EMESH, "gmsh: " + path + " is a binary .msh; write it with Mesh.Binary = 0");
    if (!(std::abs(version - 2.2) < 1e-9 || version >= 4.0))
        fail(CFG_EMESH, "gmsh: format '" + std::string(fv[0]) + "' is not supported (ASCII 2.2 and 4.1 are)");

    // physical names of surfaces (dim 2)
    std::map<long, std::string> physicalNames;
    {
        Section s = f.section("PhysicalNames", path, false);
        if (s.found())
        {
            const long n = toInt(s.take()[0], "$PhysicalNames");
            for (long i = 0; i < n; ++i)
            {
                const Row& t = s.take();
                if (t.size() < 3) fail(CFG_EMESH, "gmsh: malformed $PhysicalNames entry");
                const long dim = toInt(t[0], "$PhysicalNames");
                const long tag = toInt(t[1], "$PhysicalNames");
                std::string name;
                for (size_t k = 2; k < t.size(); ++k) name += std::string(t[k]);
                name.erase(std::remove(name.begin(), name.end(), '"'), name.end());
                if (name.empty()) fail(CFG_EMESH, "gmsh: physical group " + std::to_string(tag) + " has no name");
                if (dim == 2) physicalNames[tag] = name;
            }
        }
    }

    // nodes, renumbered densely in ascending tag order
    std::vector<Vec> points;
    // node tag -> dense index: the sorted tags, searched unless they run 1..n
    std::vector<long> sortedTags;
    bool denseTags = true;
    auto tagIndex = [&](long tag, int64_t& index) {
        if (denseTags)
        {
            if (tag < 1 || tag > static_cast<long>(sortedTags.size())) return false;
            index = tag - 1;
            return true;
        }
        const auto it = std::lower_bound(sortedTags.begin(), sortedTags.end(), tag);
        if (it == sortedTags.end() || *it != tag) return false;
        index = static_cast<int64_t>(it - sortedTags.begin());
        return true;
    };
    {
        Section sec = f.section("Nodes", path, true);
        if (!sec.found()) fail(CFG_EMESH, "gmsh: " + path + " has an empty $Nodes section");
        std::vector<std::pair<long, Vec>> rec;
        long declared = 0;
        auto coords = [&](const Row& t) {
            if (t.size() < 3) fail(CFG_EMESH, "gmsh: malformed node coordinate in $Nodes");
            return Vec{toDouble(t[0], "$Nodes"), toDouble(t[1], "$Nodes"), toDouble(t[2], "$Nodes")};
        };
        if (version < 3.0)
        {
            declared = toInt(sec.take()[0], "$Nodes");
            const long avail = std::max(0L, std::min(declared, static_cast<long>(sec.remaining())));
            rec.resize(static_cast<size_t>(avail));
            parallelChunks(avail, 1 << 14, [&](int64_t b, int64_t e) {
                for (int64_t i = b; i < e; ++i)
                {
                    const Row& t = sec.peek(static_cast<size_t>(i));
                    if (t.size() < 4) fail(CFG_EMESH, "gmsh: malformed node line in " + path);
                    rec[static_cast<size_t>(i)] = {toInt(t[0], "$Nodes"), Vec{toDouble(t[1], "$Nodes"), toDouble(t[2], "$Nodes"),
                                                                            toDouble(t[3], "$Nodes")}};
                }
            });
            sec.skip(static_cast<size_t>(avail));
            if (avail < declared) sec.take();  // the truncation error
        }
        else
        {
            const Row h = sec.take();
            if (h.size() < 4) fail(CFG_EMESH, "gmsh: malformed $Nodes header in " + path);
            const long blocks = toInt(h[0], "$Nodes header");
            declared = toInt(h[1], "$Nodes header");
            const long firstTag = toInt(h[2], "$Nodes header");
            for (long b = 0; b < blocks; ++b)
            {
                const Row bh = sec.take();
                if (bh.size() < 4) fail(CFG_EMESH, "gmsh: malformed $Nodes block header in " + path);
                const long num = toInt(bh[3], "$Nodes block");
                if (num <= 0) continue;
                const bool documented = bh.size() >= 6;
                const long minTag = documented ? toInt(bh[4], "$Nodes block") : firstTag;
                const long maxTag = documented ? toInt(bh[5], "$Nodes block") : firstTag;
                std::vector<long> tags;
                std::vector<Vec> xyz;
                if (documented)
                {
                    const long avail = std::min(num, static_cast<long>(sec.remaining()));
                    xyz.resize(static_cast<size_t>(avail));
                    parallelChunks(avail, 1 << 14, [&](int64_t b, int64_t e) {
                        for (int64_t i = b; i < e; ++i) xyz[static_cast<size_t>(i)] = coords(sec.peek(static_cast<size_t>(i)));
                    });
                    sec.skip(static_cast<size_t>(avail));
                    if (avail < num) sec.take();  // the truncation error
                    if (minTag != maxTag)
                    {
                        long v = 0;
                        while (static_cast<long>(tags.size()) < num && sec.takeSingleInt(v)) tags.push_back(v);
                    }
                    if (tags.empty())
                        for (long i = 0; i < num; ++i) tags.push_back(minTag + i);
                }
                else
                {
                    long v = 0;
                    while (static_cast<long>(tags.size()) < num && sec.takeSingleInt(v)) tags.push_back(v);
                    const bool tagged = static_cast<long>(tags.size()) == num;
                    for (long i = 0; i < num; ++i) xyz.push_back(coords(sec.take()));
                    if (!tagged) tags.assign(static_cast<size_t>(num), 0);
                }
                for (size_t i = 0; i < xyz.size(); ++i) rec.push_back({tags[i], xyz[i]});
            }
        }
        if (static_cast<long>(rec.size()) != declared)
            fail(CFG_EMESH, "gmsh: $Nodes declares " + std::to_string(declared) + " nodes, " +
                                std::to_string(rec.size()) + " were read from " + path +
                                " (unsupported node layout?)");
        // untagged nodes take the smallest unused positive tags in file order
        bool anyUntagged = false;
        for (const auto& r : rec) anyUntagged = anyUntagged || r.first <= 0;
        if (anyUntagged)
        {
            std::set<long> used;
            for (const auto& r : rec)
                if (r.first > 0) used.insert(r.first);
            long cand = 1;
            for (auto& r : rec)
            {
                if (r.first > 0) continue;
                while (used.count(cand)) ++cand;
                r.first = cand;
                used.insert(cand);
            }
        }
        const auto byTag = [](const auto& a, const auto& b) { return a.first < b.first; };
        if (!std::is_sorted(rec.begin(), rec.end(), byTag)) std::stable_sort(rec.begin(), rec.end(), byTag);
        points.reserve(rec.size());
        sortedTags.reserve(rec.size());
        for (const auto& r : rec)
        {
            if (!sortedTags.empty() && sortedTags.back() == r.first)
                fail(CFG_EMESH, "gmsh: duplicate node tag " + std::to_string(r.first) + " in " + path);
            denseTags = denseTags && r.first == static_cast<long>(sortedTags.size()) + 1;
            sortedTags.push_back(r.first);
            points.push_back(r.second);
        }
    }

    // entity -> physical tag of surfaces (4.x)
    std::map<long, long> entityPhysical;
    if (version >= 3.0)
    {
        Section en = f.section("EntityNames", path, false);
        if (en.found())
        {
            const long n = toInt(en.take()[0], "$EntityNames");
            for (long i = 0; i < n; ++i)
            {
                const Row& t = en.take();
                if (t.size() < 4) fail(CFG_EMESH, "gmsh: malformed $EntityNames entry");
                if (toInt(t[0], "$EntityNames") == 2) entityPhysical[toInt(t[1], "$EntityNames")] = toInt(t[2], "$EntityNames");
            }
        }
        Section es = f.section("Entities", path, false);
        if (es.found())
        {
            const Row h = es.take();
            if (h.size() < 4) fail(CFG_EMESH, "gmsh: malformed $Entities header");
            for (int dim = 0; dim < 4; ++dim)
            {
                const long n = toInt(h[static_cast<size_t>(dim)], "$Entities");
                for (long i = 0; i < n; ++i)
                {
                    const Row& t = es.take();
                    if (dim != 2) continue;
                    if (t.size() < 8) fail(CFG_EMESH, "gmsh: malformed $Entities surface line");
                    const long tag = toInt(t[0], "$Entities");
                    const long nPhys = toInt(t[7], "$Entities");
                    if (nPhys > 0)
                    {
                        if (t.size() < 9) fail(CFG_EMESH, "gmsh: malformed $Entities surface line");
                        entityPhysical[tag] = toInt(t[8], "$Entities");
                    }
                }
            }
        }
    }

    // elements: volumes into cells, surfaces into physical names
    std::vector<int32_t> types;
    std::vector<int64_t> offsets{0}, verts;
    SurfaceNames surfaceNames;
    {
        Section sec = f.section("Elements", path, true);
        if (!sec.found()) fail(CFG_EMESH, "gmsh: " + path + " has an empty $Elements section");
        // rows decode independently (in parallel); their cells and surface
        // names are then committed in file order
        struct Decoded
        {
            int type, npn;
            long physical;
            int64_t nodes[8];
        };
        auto decode = [&](int type, long physical, const Row& t, size_t first, int npn, Decoded& d) {
            d.type = type;
            d.npn = npn;
            d.physical = physical;
            for (int k = 0; k < npn; ++k)
            {
                const long tag = toInt(t[first + static_cast<size_t>(k)], "$Elements");
                if (!tagIndex(tag, d.nodes[k]))
                    fail(CFG_EMESH, "gmsh: an element refers to node " + std::to_string(tag) +
                                        ", which $Nodes does not define");
            }
            if (std::unique(d.nodes, d.nodes + npn) != d.nodes + npn)
                fail(CFG_EMESH, "gmsh: element " + std::to_string(type) + " repeats a node");
            if (type == 7) fail(CFG_EMESH, "gmsh: pyramid elements are not supported");
        };
        auto commit = [&](const std::vector<Decoded>& dec) {
            for (const Decoded& d : dec)
            {
                if (d.type == 2 || d.type == 3)
                {
                    const auto nit = physicalNames.find(d.physical);
                    if (nit == physicalNames.end()) continue;
                    // a triangle or quad: npn is 3 or 4 here
                    std::array<int64_t, 5> key{-1, -1, -1, -1, -1};
                    for (int k = 0; k < d.npn; ++k) key[static_cast<size_t>(k)] = d.nodes[k];
                    std::sort(key.begin(), key.begin() + (d.type == 2 ? 3 : 4));
                    surfaceNames.emplace(key, nit->second);
                }
                else if (d.type == 4 || d.type == 5 || d.type == 6)
                {
                    types.push_back(d.type);
                    verts.insert(verts.end(), d.nodes, d.nodes + d.npn);
                    offsets.push_back(static_cast<int64_t>(verts.size()));
                }
            }
        };
        if (version < 3.0)
        {
            const long declared = toInt(sec.take()[0], "$Elements");
            const long avail = std::max(0L, std::min(declared, static_cast<long>(sec.remaining())));
            std::vector<Decoded> dec(static_cast<size_t>(avail));
            parallelChunks(avail, 1 << 13, [&](int64_t b, int64_t e) {
                for (int64_t i = b; i < e; ++i)
                {
                    const Row& t = sec.peek(static_cast<size_t>(i));
                    if (t.size() < 3) fail(CFG_EMESH, "gmsh: malformed element line in " + path);
                    const int type = static_cast<int>(toInt(t[1], "$Elements"));
                    const int npn = nodesPerElement(type);
                    if (npn <= 0)
                        fail(CFG_EMESH, "gmsh: element type " + std::to_string(type) + " in " + path +
                                            " is not a first-order element; mesh with Linear order");
                    const long nTags = toInt(t[2], "$Elements");
                    if (static_cast<long>(t.size()) < 3 + nTags + npn)
                        fail(CFG_EMESH, "gmsh: truncated element line in " + path);
                    const long physical = nTags > 0 ? toInt(t[3], "$Elements") : 0;
                    decode(type, physical, t, static_cast<size_t>(3 + nTags), npn, dec[static_cast<size_t>(i)]);
                }
            });
            sec.skip(static_cast<size_t>(avail));
            if (avail < declared) sec.take();  // the truncation error
            types.reserve(dec.size());
            offsets.reserve(dec.size() + 1);
            verts.reserve(8 * dec.size());
            commit(dec);
        }
        else
        {
            const Row h = sec.take();
            if (h.size() < 4) fail(CFG_EMESH, "gmsh: malformed $Elements header in " + path);
            const long blocks = toInt(h[0], "$Elements header");
            const long declared = toInt(h[1], "$Elements header");
            long read = 0;
            for (long b = 0; b < blocks; ++b)
            {
                const Row bh = sec.take();
                if (bh.size() < 4) fail(CFG_EMESH, "gmsh: malformed $Elements block header in " + path);
                const long entityTag = toInt(bh[1], "$Elements block");
                const int type = static_cast<int>(toInt(bh[2], "$Elements block"));
                const long num = toInt(bh[3], "$Elements block");
                const int npn = nodesPerElement(type);
                if (npn <= 0)
                    fail(CFG_EMESH, "gmsh: element type " + std::to_string(type) + " in " + path +
                                        " is not a first-order element; mesh with Linear order");
                const auto pit = entityPhysical.find(entityTag);
                const long physical = pit != entityPhysical.end() ? pit->second : 0;
                const long avail = std::max(0L, std::min(num, static_cast<long>(sec.remaining())));
                // the first line fixes whether the lines carry the element tag
                bool tagged = false;
                if (avail > 0)
                {
                    const long width = static_cast<long>(sec.peek(0).size());
                    if (width == npn + 1) tagged = true;
                    else if (width != npn)
                        fail(CFG_EMESH, "gmsh: element line with " + std::to_string(width) + " entries, expected " +
                                            std::to_string(npn) + " or " + std::to_string(npn + 1));
                }
                std::vector<Decoded> dec(static_cast<size_t>(avail));
                parallelChunks(avail, 1 << 13, [&](int64_t lo, int64_t hi) {
                    for (int64_t i = lo; i < hi; ++i)
                    {
                        const Row& t = sec.peek(static_cast<size_t>(i));
                        if (static_cast<long>(t.size()) != npn + (tagged ? 1 : 0))
                            fail(CFG_EMESH, "gmsh: inconsistent element line width in " + path);
                        decode(type, physical, t, tagged ? 1 : 0, npn, dec[static_cast<size_t>(i)]);
                    }
                });
                sec.skip(static_cast<size_t>(avail));
                read += avail;
                if (avail < num) sec.take();  // the truncation error
                commit(dec);
            }
            if (read != declared)
                fail(CFG_EMESH, "gmsh: $Elements declares " + std::to_string(declared) + " elements, " +
                                    std::to_string(read) + " were read from " + path +
                                    " (unsupported element layout?)");
        }
    }
    if (types.empty()) fail(CFG_EMESH, "gmsh: " + path + " has no volume elements");
    return meshFromCells(points, types, offsets, verts, surfaceNames, patchTypes);
}

}  // namespace cfg
